"""The oracle's restatement of compare.py (the reference's curve-comparison
metric) reproduces the values the reference's own runs printed in
test/test23/test-results/perf-comp-acc.txt, from the committed curves."""
from __future__ import annotations

import numpy as np
import pytest

CASES = [(m, dz) for m in (4, 5, 6, 7) for dz in ("0.68", "0.1", "0.022")]


@pytest.mark.parametrize("method,dz", CASES)
def test_compare_reproduces_printed_rows(golden, oracle_mod, method, dz):
    acc = np.load(golden / "test23" / "accurate.npz")
    perf = np.load(golden / "test23" / f"perf-{method}-{dz}.npz")
    rows = acc[f"comp-{method}-{dz}"]
    got = oracle_mod.compare_curves(perf["f2"], acc["f2"])
    np.testing.assert_allclose(rows[:, 0], perf["angle"], atol=1e-12)
    # the script printed 16 significant digits
    np.testing.assert_allclose(got, rows[:, 1:], rtol=1e-12, atol=0)
