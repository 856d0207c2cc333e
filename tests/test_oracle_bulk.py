"""The oracle's bulk solve (bulk.txt -> bulkP.b) against the reference's records.

The committed bulkP.b files were written by the original code (netlib
eigensolver + Gauss-Jordan), so the reflection-matrix records agree to
rounding (measured 2e-12 for test23, 2e-9 for the worst test47 record); the
header records must be byte-identical.
"""
from __future__ import annotations

import struct

import numpy as np
import pytest


def records(path):
    b = open(path, "rb").read()
    out, p = [], 0
    while p < len(b):
        n = struct.unpack("<i", b[p:p + 4])[0]
        out.append(b[p + 4:p + 4 + n])
        p += 8 + n
    return out


@pytest.mark.parametrize("case,tol", [("test23", 1e-10), ("test47", 1e-8)])
def test_bulk_records(golden, oracle_mod, tmp_path, case, tol):
    d = golden / case
    out = tmp_path / "bulkP.b"
    oracle_mod.bulk_run(d / "bulk.txt", out)
    mine, ref = records(out), records(d / "bulkP.b")
    assert len(mine) == len(ref)
    nhdr = 16  # 8 fixed + 2 per element (1) + 1 per atom (2) + 4 domain records
    for i in range(nhdr):
        assert mine[i] == ref[i], f"header record {i}"
    worst = 0.0
    for x, y in zip(mine[nhdr:], ref[nhdr:]):
        xa, ya = np.frombuffer(x, np.complex128), np.frombuffer(y, np.complex128)
        worst = max(worst, np.abs(xa - ya).max() / max(np.abs(ya).max(), 1e-300))
    assert worst <= tol, worst
