"""The oracle's rocking-curve convolution against the reference's own samples:
convolution.txt files written by make_convolution.py from the sample rocking
curves (printed with 6 and 9 significant digits)."""
from __future__ import annotations

import numpy as np
import pytest


@pytest.mark.parametrize("name,tol", [("ge001", 2e-6), ("t4al", 5e-6)])
def test_convolution_matches_reference_sample(golden, oracle_mod, name, tol):
    d = np.load(golden / f"conv-{name}.npz")
    got = oracle_mod.rocking_convolution(d["angle"], d["f2"], 0.5)
    np.testing.assert_allclose(d["conv_angle"], d["angle"])
    err = np.abs(got - d["conv"]).max() / np.abs(d["conv"]).max()
    assert err <= tol, err
