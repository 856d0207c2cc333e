"""CUDA-graph replay of resident solves: the first solve of a problem runs its
launches directly, the second is captured into a graph, later ones replay it.
Every one of them must give the same intensities as direct launches, bit for
bit: the same kernels run in the same order on the same buffers."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from trhepd_opt_b200 import build, native
    build.build()
    c = native.Context(0)
    yield c
    c.close()


def _resident(ctx, tmp_path, s):
    from trhepd_opt_b200 import bulkfile, surface
    s.write(tmp_path)
    bulkfile.write_bulkp(s, tmp_path / "bulkP.b")
    sp = surface.SurfaceProblem(ctx, tmp_path / "bulkP.b", tmp_path / "surf.txt", s.surface_dz,
                                s.int_method)
    return sp, sp.resident()


@pytest.mark.parametrize("precision", [0, 1, 2], ids=["fp64", "bf16", "int8"])
@pytest.mark.parametrize("method", [5, 7, 2], ids=["rkn4", "rk4", "magnus4"])
def test_graph_replay_equals_direct(ctx, tmp_path, precision, method):
    from trhepd_opt_b200 import generator, native
    if method == 2 and precision:
        pytest.skip("the Magnus integrators run in plain FP64 only")
    s = generator.small23()
    s.int_method = method
    sp, rp = _resident(ctx, tmp_path, s)
    ctx.set_option(native.OPT_GRAPHS, 0)
    rp.solve(precision)
    _, direct = rp.fetch()
    launches = ctx.last_stats()["launches"]
    ctx.set_option(native.OPT_GRAPHS, 1)
    out = []
    for _ in range(4):  # direct, capture + replay, replay, replay
        rp.solve(precision)
        out.append(rp.fetch()[1])
        assert ctx.last_stats()["launches"] == launches
    for f2 in out:
        assert np.array_equal(f2, direct)


def test_graph_follows_option_changes(ctx, tmp_path):
    """A changed option (slices) between solves means a new capture."""
    from trhepd_opt_b200 import generator, native
    sp, rp = _resident(ctx, tmp_path, generator.small23())
    ref = {}
    ctx.set_option(native.OPT_GRAPHS, 0)
    for S in (3, 4):
        ctx.set_option(native.OPT_SPLIT_SLICES, S)
        rp.solve(native.SPLIT_INT8)
        ref[S] = rp.fetch()[1]
    ctx.set_option(native.OPT_GRAPHS, 1)
    for S in (3, 3, 3, 4, 4, 4, 3, 3):
        ctx.set_option(native.OPT_SPLIT_SLICES, S)
        rp.solve(native.SPLIT_INT8)
        assert np.array_equal(rp.fetch()[1], ref[S])
    ctx.set_option(native.OPT_SPLIT_SLICES, 4)
    assert not np.array_equal(ref[3], ref[4])
