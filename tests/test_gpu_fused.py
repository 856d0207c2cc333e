"""Fused small-beam integration (one CTA per angle, state in shared memory)
against the stacked path (one launch per stage), the oracle and the reference's
outputs.  Both are the same FP64 arithmetic in a different summation order, so
they agree to rounding: 1e-10 of the row maximum on these short cases."""
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
    yield c
    c.close()


def _resident(ctx, tmp_path, s):
    from trhepd_opt_b200 import bulkfile, surface
    s.write(tmp_path)
    bulkfile.write_bulkp(s, tmp_path / "bulkP.b")
    sp = surface.SurfaceProblem(ctx, tmp_path / "bulkP.b", tmp_path / "surf.txt", s.surface_dz,
                                s.int_method)
    return sp, sp.resident()


@pytest.mark.parametrize("policy", [0, 1], ids=["gershgorin", "growth"])
@pytest.mark.parametrize("n,method", [(13, 5), (23, 5), (23, 6), (40, 5), (64, 5)])
def test_fused_matches_stacked(ctx, tmp_path, n, method, policy):
    from trhepd_opt_b200 import generator, native
    s = generator.dense(n, n_angles=9, region=3.0) if n != 23 else generator.small23()
    s.int_method = method
    sp, rp = _resident(ctx, tmp_path, s)
    ctx.set_option(native.OPT_RENORM_POLICY, policy)
    try:
        ctx.set_option(native.OPT_FUSED_MAX_N, 0)
        rp.solve(native.FP64)
        _, stacked = rp.fetch()
        ctx.set_option(native.OPT_FUSED_MAX_N, 64)
        rp.solve(native.FP64)
        _, fused = rp.fetch()
        assert ctx.last_stats()["launches"] < 40  # boundary kernels plus one integration
    finally:
        ctx.set_option(native.OPT_RENORM_POLICY, 0)
        ctx.set_option(native.OPT_FUSED_MAX_N, 64)
    assert np.isfinite(fused).all()
    abs_err, rel = spot_errors(fused, stacked)
    assert abs_err <= 1e-10, abs_err
    assert rel <= 1e-8, rel


def test_fused_against_oracle(ctx, tmp_path, oracle_mod):
    from trhepd_opt_b200 import generator, native
    s = generator.dense(47, n_angles=6, region=3.0, seed=4)
    s.write(tmp_path)
    from trhepd_opt_b200 import bulkfile
    bulkfile.write_bulkp(s, tmp_path / "bulkP.b")
    f2, _ = ctx.surf_run(tmp_path / "bulkP.b", tmp_path / "surf.txt", s.surface_dz, 5,
                         native.FP64)
    ref, _, _ = oracle_mod.Surface(tmp_path / "bulkP.b", tmp_path / "surf.txt", s.surface_dz,
                                   5).solve()
    abs_err, rel = spot_errors(f2, ref)
    assert abs_err <= 1e-10, abs_err
    assert rel <= 1e-8, rel
