"""The oracle's int_method 8 (rk4_intgs, sim-trhepd-rheed/src/surf_rk.f90:93-156)
against the reference's committed int_method 7 outputs.

Method 8 runs the RK4 stages of method 7 (the same rk4_int_init table and step)
and re-orthogonalises [q; p] by CholeskyQR when a power estimate of its squared
norm exceeds 1e2 (matgs.f90:5-35, matcomp.f90:530-594).  A right multiplication of
[q; p] leaves f = p q^{-1} unchanged, so the reference's method-7 outputs pin
method 8 up to rounding; the reference ships no method-8 outputs of its own.
Measured: 1.9e-11 relative on every spot of test23 at dz 0.68, ~1e-13 elsewhere.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import spot_errors


@pytest.mark.parametrize("case,dz", [("test23", "0.68"), ("test23", "0.1"), ("test47", "0.22")])
def test_oracle_method8_matches_reference_rk4(golden, oracle_mod, case, dz):
    d = golden / case
    ref = np.load(d / f"perf-7-{dz}.npz")
    S = oracle_mod.Surface(d / "bulkP.b", d / "surf.txt", float(dz), 8)
    f2, ang, renorm = S.solve()
    np.testing.assert_allclose(ang, ref["angle"], rtol=0, atol=5e-5)
    abs_err, rel_err = spot_errors(f2, ref["f2"])
    assert abs_err <= 1e-10, abs_err
    assert rel_err <= 1e-9, rel_err
    assert np.asarray(renorm).max() > 0  # CholeskyQR steps were taken


def test_oracle_method8_differs_from_method7(golden, oracle_mod):
    d = golden / "test23"
    f8, _, r8 = oracle_mod.Surface(d / "bulkP.b", d / "surf.txt", 0.1, 8).solve()
    f7, _, r7 = oracle_mod.Surface(d / "bulkP.b", d / "surf.txt", 0.1, 7).solve()
    assert not np.array_equal(f7, f8)
    assert not np.array_equal(np.asarray(r7), np.asarray(r8))
