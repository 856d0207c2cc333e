"""Rocking-curve convolution on the GPU (trhepd_rocking_convolution,
trhepd_problem_convolve) against the reference's own convolution samples and
against the oracle's restatement on a solved two-azimuth problem."""
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


@pytest.mark.parametrize("name,tol", [("ge001", 2e-6), ("t4al", 5e-6)])
def test_convolution_matches_reference_sample(ctx, golden, name, tol):
    d = np.load(golden / f"conv-{name}.npz")
    got = ctx.rocking_convolution(d["angle"], d["f2"], 0.5)
    err = np.abs(got - d["conv"]).max() / np.abs(d["conv"]).max()
    assert err <= tol, err


def test_problem_convolution_matches_oracle(ctx, tmp_path, oracle_mod):
    """Two azimuths: each block of the inner scan is convolved alone."""
    from trhepd_opt_b200 import bulkfile, generator, native, surface
    s = generator.batch47()
    s.write(tmp_path)
    bulkfile.write_bulkp(s, tmp_path / "bulkP.b")
    sp = surface.SurfaceProblem(ctx, tmp_path / "bulkP.b", tmp_path / "surf.txt", s.surface_dz,
                                s.int_method)
    rp = sp.resident()
    rp.solve(native.FP64)
    ang, f2 = rp.fetch()
    got = rp.convolve(0.5)
    nblocks = 2
    ref = oracle_mod.rocking_convolution(ang, f2, 0.5, scan=len(ang) // nblocks)
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err <= 1e-13, err
    rp.close()
    sp.close()


def test_convolution_rejects_single_angle(ctx):
    from trhepd_opt_b200 import native
    with pytest.raises(native.TrhepdError):
        ctx.rocking_convolution(np.zeros(1), np.zeros((1, 3)), 0.5)
