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


def test_bulk_ge_sample(golden, oracle_mod, tmp_path):
    """The reference's Ge(001) sample (Z = 32, plane group 6, one beam, 70 angles):
    the header records, which carry the element's scattering-factor coefficients,
    are byte-identical and the records agree to rounding."""
    d = golden / "ge001"
    out = tmp_path / "bulkP.b"
    oracle_mod.bulk_run(d / "bulk.txt", out)
    mine, ref = records(out), records(d / "bulkP.b")
    assert len(mine) == len(ref) == 16 + 70
    for i in range(16):
        assert mine[i] == ref[i], f"header record {i}"
    for x, y in zip(mine[16:], ref[16:]):
        xa, ya = np.frombuffer(x, np.complex128), np.frombuffer(y, np.complex128)
        assert np.abs(xa - ya).max() <= 1e-12 * np.abs(ya).max()


def test_bulk_electron_mode(golden, oracle_mod, tmp_path):
    """Electrons (bulk.exe with ep = 'E', bulkm.f90:21-24): inegpos = 0 in the
    header and the scattering-factor coefficients without the positron sign flip
    (bulkio.f90:74); the Python header writer agrees byte for byte."""
    import struct as st

    from trhepd_opt_b200 import bulkfile, generator
    d = golden / "test23"
    oracle_mod.set_electron(True)
    try:
        oracle_mod.bulk_run(d / "bulk.txt", tmp_path / "e.b")
    finally:
        oracle_mod.set_electron(False)
    oracle_mod.bulk_run(d / "bulk.txt", tmp_path / "p.b")
    e, p = records(tmp_path / "e.b"), records(tmp_path / "p.b")
    assert st.unpack("<10i", e[1])[0] == 0 and st.unpack("<10i", p[1])[0] == 1
    ae, ap = np.frombuffer(e[8], np.float64), np.frombuffer(p[8], np.float64)
    np.testing.assert_array_equal(ae[:4], -ap[:4])        # a(1:nabr), flipped for positrons
    np.testing.assert_array_equal(ae[4:], ap[4:])         # sap, b
    assert any(x != y for x, y in zip(e[16:], p[16:]))    # different reflection records
    s = generator.small23()
    bulk_txt, _ = s.write(tmp_path / "s")
    oracle_mod.set_electron(True)
    try:
        oracle_mod.bulk_run(bulk_txt, tmp_path / "s" / "oracle.b")
    finally:
        oracle_mod.set_electron(False)
    bulkfile.write_bulkp(s, tmp_path / "s" / "py.b", electron=True)
    mine, ref = records(tmp_path / "s" / "py.b"), records(tmp_path / "s" / "oracle.b")
    assert len(mine) == len(ref)
    for i in range(16):
        assert mine[i] == ref[i], f"header record {i}"
