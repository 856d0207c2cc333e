"""Candidate-structure batches (trhepd_batch_solve): small-beam problems of
different beam counts, jitters and angle grids share one fused launch, a larger
problem runs after them; every problem's intensities must equal its solve on
its own (the same per-element arithmetic: 1e-12 of the row maximum)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import spot_errors

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from trhepd_opt_b200 import build, native
    build.build()
    c = native.Context(0)
    c.set_option(native.OPT_RENORM_POLICY, 1)
    yield c
    c.close()


def _resident(ctx, d, s):
    from trhepd_opt_b200 import bulkfile, surface
    s.write(d)
    bulkfile.write_bulkp(s, d / "bulkP.b")
    sp = surface.SurfaceProblem(ctx, d / "bulkP.b", d / "surf.txt", s.surface_dz, s.int_method)
    return sp, sp.resident()


def _structures():
    from trhepd_opt_b200 import generator
    base23 = generator.small23()
    base47 = generator.dense(47, n_angles=7, region=3.0, seed=5)
    out = [base23, generator.jitter(base23, 0.1, 1), base47, generator.jitter(base47, 0.15, 2),
           generator.dense(23, n_angles=11, region=2.5, seed=8),
           generator.dense(95, n_angles=5, region=2.0, seed=9)]
    out[4].int_method = 6  # an RKN-6 problem takes its own fused launch
    return out


@pytest.mark.parametrize("policy", [0, 1], ids=["gershgorin", "growth"])
def test_batch_equals_individual(ctx, tmp_path, policy):
    from trhepd_opt_b200 import native, surface
    ctx.set_option(native.OPT_RENORM_POLICY, policy)
    probs = []
    for k, s in enumerate(_structures()):
        d = tmp_path / f"s{k}"
        probs.append(_resident(ctx, d, s))
    alone = []
    for sp, rp in probs:
        rp.solve(native.FP64)
        alone.append(rp.fetch()[1])
    for _ in range(2):  # twice: the larger problem's second solve is a graph replay
        surface.solve_batch(ctx, [rp for _, rp in probs], native.FP64)
        st = ctx.last_stats()
        assert st["device_ms"] > 0 and st["stage_products"] > 0
        for (sp, rp), ref in zip(probs, alone):
            _, got = rp.fetch()
            assert np.isfinite(got).all()
            abs_err, _ = spot_errors(got, ref)
            assert abs_err <= 1e-12, (rp.nb, abs_err)
    for sp, rp in probs:
        rp.close()
        sp.close()
    ctx.set_option(native.OPT_RENORM_POLICY, 1)


def test_batch_split_form_on_the_larger_problem(ctx, tmp_path):
    """In a split-precision batch the fused problems stay FP64 (exact) and the
    larger one runs the INT8 form: equal to its own INT8 solve."""
    from trhepd_opt_b200 import native, surface
    probs = [_resident(ctx, tmp_path / f"s{k}", s) for k, s in enumerate(_structures())]
    ref = []
    for sp, rp in probs:
        rp.solve(native.FP64 if rp.nb <= 64 else native.SPLIT_INT8)
        ref.append(rp.fetch()[1])
    surface.solve_batch(ctx, [rp for _, rp in probs], native.SPLIT_INT8)
    for (sp, rp), r in zip(probs, ref):
        _, got = rp.fetch()
        assert spot_errors(got, r)[0] <= 1e-12
    for sp, rp in probs:
        rp.close()
        sp.close()


def test_batch_rejects_empty(ctx):
    from trhepd_opt_b200 import native, surface
    with pytest.raises(native.TrhepdError):
        surface.solve_batch(ctx, [], native.FP64)


@pytest.mark.parametrize("precision", [0, 2], ids=["fp64", "int8"])
def test_stacked_candidates_equal_individual(ctx, tmp_path, precision):
    """Candidates of one base structure (same beams, slices, angle grid) are
    integrated as one stacked solve, every row tile with its own stage matrix:
    each must equal its own solve.  A structure with another angle grid is
    solved on its own, a small one in the fused launch."""
    from trhepd_opt_b200 import generator, native, surface
    base = generator.dense(95, n_angles=5, region=2.0, seed=12)
    structs = [generator.jitter(base, 0.1, k) for k in range(3)]
    structs.append(generator.dense(95, n_angles=4, region=2.0, seed=13))
    structs.append(generator.jitter(generator.small23(), 0.1, 5))
    probs = [_resident(ctx, tmp_path / f"s{k}", s) for k, s in enumerate(structs)]
    ref = []
    for sp, rp in probs:
        rp.solve(native.FP64 if rp.nb <= 64 else precision)
        ref.append(rp.fetch()[1])
    surface.solve_batch(ctx, [rp for _, rp in probs], precision)
    for (sp, rp), r in zip(probs, ref):
        _, got = rp.fetch()
        assert np.isfinite(got).all()
        assert spot_errors(got, r)[0] <= 1e-12, rp.nb
    for sp, rp in probs:
        rp.close()
        sp.close()
