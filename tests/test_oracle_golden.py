"""The CPU oracle against the reference's own committed outputs.

Fixtures (tests/golden/, made by make_golden.py from the reference's
test/<case>/test-results/perf-<method>-<dz>.txt, 15 significant digits) pin
the oracle before it is trusted as the checker of the CUDA path.  The
tolerance is the plain FP64 bar: 1e-9 relative on every spot at least 1e-6 of
its row's maximum, and 1e-10 of the row maximum on every spot.  The remaining
differences come from BLAS/LAPACK rounding (MKL in the reference, OpenBLAS
here).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import spot_errors

CASES = [("test23", m, dz) for m in (4, 5, 6, 7) for dz in ("0.68", "0.1", "0.022")]
CASES += [("test47", 5, "0.68"), ("test47", 6, "0.68"), ("test47", 5, "0.22"),
          ("test47", 7, "0.22"), ("test521", 5, "0.68")]


@pytest.mark.parametrize("case,method,dz", CASES)
def test_oracle_matches_reference_output(golden, oracle_mod, case, method, dz):
    d = golden / case
    ref = np.load(d / f"perf-{method}-{dz}.npz")
    S = oracle_mod.Surface(d / "bulkP.b", d / "surf.txt", float(dz), method)
    f2, ang, _ = S.solve()
    np.testing.assert_allclose(ang, ref["angle"], rtol=0, atol=5e-5)
    abs_err, rel_err = spot_errors(f2, ref["f2"])
    assert abs_err <= 1e-10, abs_err
    assert rel_err <= 1e-9, rel_err


def test_oracle_writes_reference_format(golden, oracle_mod, tmp_path):
    """Rocking-curve file layout (header, 400I4 beam lines, E23.15 rows with
    format reversion and trailing comma) matches the reference's file."""
    d = golden / "test23"
    S = oracle_mod.Surface(d / "bulkP.b", d / "surf.txt", 0.68, 5)
    out = tmp_path / "surf-bulkP.s"
    S.write(out)
    mine = out.read_text().split("\n")
    import trhepd_opt_b200.formats as F
    ang, f2, hdr = F.read_rocking_curves(out)
    ref = np.load(d / "perf-5-0.68.npz")
    assert hdr["nb"] == 23 and f2.shape == ref["f2"].shape
    assert mine[0] == "#azimuths,g-angles,beams" and mine[1] == "   1  69  23"
    assert all(len(l) == 565 for l in mine[4:4 + 69])


def test_oracle_wide_rows(golden, oracle_mod, tmp_path):
    """nb = 521 rows span three lines (200 + 200 + 121 values)."""
    d = golden / "test521"
    S = oracle_mod.Surface(d / "bulkP.b", d / "surf.txt", 0.68, 5)
    out = tmp_path / "s.s"
    S.write(out)
    L = out.read_text().split("\n")
    assert [len(x) for x in L[3:9]] == [1600, 1600, 968, 4812, 4800, 2905]
    assert L[7].startswith(",") and L[8].endswith(",")
