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


def test_bulk_conditioning(golden, oracle_mod, tmp_path):
    """The reference's bulk records are well-conditioned on its own structures and
    not on strongly evanescent synthetic cells: a 2^-50 rescale of the slice
    potentials moves test23's records by < 1e-10 and a synthetic 2x2 cell's by
    > 1e-4 (the bound the GPU bulk tests derive their tolerances from)."""
    from trhepd_opt_b200 import generator

    def sens(bulk_txt, d):
        d.mkdir(exist_ok=True)
        oracle_mod.set_bulk_scale(1.0)
        oracle_mod.bulk_run(bulk_txt, d / "a.b")
        oracle_mod.set_bulk_scale(1.0 + 2.0 ** -50)
        try:
            oracle_mod.bulk_run(bulk_txt, d / "b.b")
        finally:
            oracle_mod.set_bulk_scale(1.0)
        worst = 0.0
        for x, y in zip(records(d / "a.b"), records(d / "b.b")):
            if x != y:
                xa, ya = np.frombuffer(x, np.complex128), np.frombuffer(y, np.complex128)
                worst = max(worst, float(np.abs(xa - ya).max() / np.abs(xa).max()))
        return worst

    assert sens(golden / "test23" / "bulk.txt", tmp_path / "g") < 1e-10
    s = generator.dense(23, seed=5, n_angles=7, region=4.0, dz=0.02)
    bulk_txt, _ = s.write(tmp_path / "s")
    assert sens(bulk_txt, tmp_path / "s") > 1e-4

