"""GPU bulk solve (trhepd_bulk_run: bulk.txt -> bulkP.b) against the reference.

The reference's bulkP.b files (tests/golden/*/bulkP.b, written by the original
eigen-decomposition path of trmat, sim-trhepd-rheed/src/bulk.f90:130-264) pin the
reflection records; the GPU builds the slice transfer matrix from the matrix
cosine/sine series instead of eigenvectors, so records agree to rounding of
the two constructions, amplified by the conditioning of the layer recursion.
Header records must be byte-identical.  Synthetic structures are checked against
the oracle's restatement, with bounds set by the oracle's own rounding
sensitivity (a 2^-50 rescale of the potential).
"""
from __future__ import annotations

import struct

import numpy as np
import pytest

from conftest import spot_errors

pytestmark = pytest.mark.gpu


def records(path):
    b = open(path, "rb").read()
    out, p = [], 0
    while p < len(b):
        n = struct.unpack("<i", b[p:p + 4])[0]
        assert struct.unpack("<i", b[p + 4 + n:p + 8 + n])[0] == n
        out.append(b[p + 4:p + 4 + n])
        p += 8 + n
    return out


def compare(mine, ref):
    """(count of numeric records, worst record-relative difference); every
    other record must be byte-identical."""
    assert len(mine) == len(ref)
    worst, nnum = 0.0, 0
    for x, y in zip(mine, ref):
        if x == y:
            continue
        assert len(x) == len(y) and len(x) % 16 == 0
        xa, ya = np.frombuffer(x, np.complex128), np.frombuffer(y, np.complex128)
        assert np.isfinite(xa).all()
        worst = max(worst, float(np.abs(xa - ya).max() / max(np.abs(ya).max(), 1e-300)))
        nnum += 1
    return nnum, worst


@pytest.fixture(scope="module")
def ctx():
    from trhepd_opt_b200 import build, native
    build.build()
    c = native.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("case,tol", [("test23", 1e-9), ("test47", 1e-8)])
def test_bulk_golden(golden, ctx, tmp_path, case, tol):
    d = golden / case
    out = tmp_path / "bulkP.b"
    st = ctx.bulk_run(d / "bulk.txt", out)
    assert st["items"] > 0 and st["layers"] >= 20
    nnum, worst = compare(records(out), records(d / "bulkP.b"))
    assert nnum > 0
    assert worst <= tol, worst


def golden_variant(src, seed: int) -> str:
    """A seeded variant of a reference bulk.txt: Debye-Waller factors, atom heights
    and glancing-angle range redrawn, beams and cell kept (such structures keep the
    layer recursion well-conditioned, unlike the synthetic cells below)."""
    rng = np.random.default_rng(seed)
    out = []
    for line in open(src).read().split("\n"):
        if "BH(I)" in line:
            b = rng.uniform(0.3, 1.0)
            line = f"{b:.4f},{b:.4f},{b:.4f}\t\t\t,BH(I),BK(I),BZ(I)"
        elif "IELM(I),ocr(I),X(I),Y(I),Z(I)" in line:
            f = line.split(",")
            f[4] = f"  {float(f[4].split()[0]) + rng.uniform(-0.1, 0.1):.5f}\t\t"
            line = ",".join(f)
        elif "BE,AZI" in line:
            f = line.split(",")
            gi = rng.uniform(0.1, 2.0)
            f[4], f[5], f[6] = f"{gi:.2f}", f"{gi + rng.integers(3, 8) * 0.3:.2f}", "0.3\t\t\t"
            line = ",".join(f)
        out.append(line)
    return "\n".join(out)


def sensitivity(oracle_mod, bulk_txt, tmp_path):
    """The oracle's records and how far each entry moves when the slice potentials
    are rescaled by 1 + 2^-50: the rounding sensitivity of the problem itself."""
    a, b = tmp_path / "oracle.b", tmp_path / "oracle_pert.b"
    oracle_mod.set_bulk_scale(1.0)
    oracle_mod.bulk_run(bulk_txt, a)
    oracle_mod.set_bulk_scale(1.0 + 2.0 ** -50)
    try:
        oracle_mod.bulk_run(bulk_txt, b)
    finally:
        oracle_mod.set_bulk_scale(1.0)
    return records(a), records(b)


@pytest.mark.parametrize("case,seed", [("test23", 1), ("test23", 2), ("test47", 1)])
def test_bulk_synthetic_vs_oracle(oracle_mod, ctx, golden, tmp_path, case, seed):
    """Seeded variants of the reference structures, tight bound (the oracle's own
    rounding sensitivity on them is below 1e-9)."""
    bulk_txt = tmp_path / "bulk.txt"
    bulk_txt.write_text(golden_variant(golden / case / "bulk.txt", seed))
    ours = tmp_path / "gpu.b"
    ctx.bulk_run(bulk_txt, ours)
    ref, pert = sensitivity(oracle_mod, bulk_txt, tmp_path)
    _, sens = compare(pert, ref)
    assert sens <= 1e-9, sens  # the case is well-conditioned
    nnum, worst = compare(records(ours), ref)
    assert nnum > 0
    assert worst <= 1e-8, worst


@pytest.mark.parametrize("n,seed", [(23, 5)])
def test_bulk_ill_conditioned_within_sensitivity(oracle_mod, ctx, tmp_path, n, seed):
    """The synthetic 2x2 cells have strongly evanescent bulk beams (decay constants
    up to ~15/A over a 3.14 A layer): the reference's own records move by up to
    O(1) under a 2^-50 rescale of the potential.  Each entry must then agree with
    the oracle within 1e-8 of its record maximum plus 64 times that entry's
    sensitivity, and entries the rescale leaves unchanged must agree tightly.
    (At N = 95 the same generator's records move by O(1) relative under the
    rescale: rounding noise that no bound can compare, so that size is left out.)"""
    from trhepd_opt_b200 import generator
    s = generator.dense(n, seed=seed, n_angles=7, region=4.0, dz=0.02)
    bulk_txt, _ = s.write(tmp_path)
    ours = tmp_path / "gpu.b"
    ctx.bulk_run(bulk_txt, ours)
    ref, pert = sensitivity(oracle_mod, bulk_txt, tmp_path)
    mine = records(ours)
    assert len(mine) == len(ref)
    nnum = 0
    for x, y, z in zip(mine, ref, pert):
        if x == y:
            continue
        assert len(x) == len(y) and len(x) % 16 == 0
        xa, ya, za = (np.frombuffer(v, np.complex128) for v in (x, y, z))
        assert np.isfinite(xa).all()
        scale = max(np.abs(ya).max(), 1e-300)
        bound = 1e-8 * scale + 64.0 * np.abs(za - ya)
        assert (np.abs(xa - ya) <= bound).all(), float((np.abs(xa - ya) / bound).max())
        nnum += 1
    assert nnum > 0


def test_bulk_then_surface(golden, ctx, oracle_mod, tmp_path):
    """surf.exe on a GPU-written bulkP.b matches surf.exe on the reference's."""
    from trhepd_opt_b200 import native, surface
    d = golden / "test23"
    ours = tmp_path / "bulkP.b"
    ctx.bulk_run(d / "bulk.txt", ours)
    a = surface.SurfaceProblem(ctx, ours, d / "surf.txt", 0.68, 5)
    b = surface.SurfaceProblem(ctx, d / "bulkP.b", d / "surf.txt", 0.68, 5)
    fa, fb = a.srfref(native.FP64)[1], b.srfref(native.FP64)[1]
    a.close()
    b.close()
    rowmax, _ = spot_errors(fa, fb)
    assert rowmax <= 1e-8, rowmax


def test_bulk_ge_sample(golden, ctx, tmp_path):
    """The reference's Ge(001) sample (Z = 32, one beam, 70 angles): header records
    byte-identical to the bulkP.b the reference wrote, records to rounding."""
    d = golden / "ge001"
    out = tmp_path / "bulkP.b"
    ctx.bulk_run(d / "bulk.txt", out)
    mine, ref = records(out), records(d / "bulkP.b")
    assert len(mine) == 16 + 70  # 70 glancing angles x 1 beam group
    for i in range(16):
        assert mine[i] == ref[i], f"header record {i}"
    nnum, worst = compare(mine, ref)
    assert worst <= 1e-10, worst


def test_bulk_test521_within_sensitivity(golden, ctx, oracle_mod, tmp_path):
    """The reference's N = 521 bulk (nh = nk = 7, 49 beam groups of up to 53 beams,
    1 angle).  Its layer recursion is ill-conditioned in the reference's own
    algorithm for the largest groups: a 2^-50 rescale of the slice potentials moves
    the oracle's records for the groups of 53, 16 and 14 beams by O(1) of their
    maximum, and the committed bulkP.b differs from the oracle there by as much, so
    those records are rounding noise in any implementation.  Headers are
    byte-identical; every record the rescale moves by less than 1e-3 of its maximum
    (the meaningful ones, 33 of the 49) agrees with the oracle within 1e-8 plus 8x
    that record's sensitivity; the others must be finite."""
    d = golden / "test521"
    ours = tmp_path / "gpu.b"
    st = ctx.bulk_run(d / "bulk.txt", ours)
    assert st["items"] == 49
    ref, pert = sensitivity(oracle_mod, d / "bulk.txt", tmp_path)
    mine, committed = records(ours), records(d / "bulkP.b")
    assert len(mine) == len(ref) == len(committed) == 16 + 49
    for i in range(16):
        assert mine[i] == committed[i], f"header record {i}"
    checked, worst = 0, 0.0
    for i in range(16, len(mine)):
        xa, ya, za = (np.frombuffer(v[i], np.complex128) for v in (mine, ref, pert))
        assert np.isfinite(xa).all()
        sc = max(np.abs(ya).max(), 1e-300)
        sens = np.abs(za - ya).max() / sc
        if sens > 1e-3:
            continue
        worst = max(worst, (np.abs(xa - ya).max() / sc) / (1e-8 + 8.0 * sens))
        checked += 1
    assert checked >= 30, checked
    assert worst <= 1.0, worst


def test_bulk_electron_matches_oracle(golden, ctx, oracle_mod, tmp_path):
    """Electron mode (TRHEPD_OPT_PARTICLE = 1, bulk.exe with ep = 'E'): bulkP.b on the
    GPU against the oracle's, then the surface solve on that file (which follows
    its inegpos) against the oracle's surface solve."""
    from trhepd_opt_b200 import native
    d = golden / "test23"
    ours, theirs = tmp_path / "bulkE.b", tmp_path / "oracleE.b"
    ctx.set_option(native.OPT_PARTICLE, 1)
    try:
        ctx.bulk_run(d / "bulk.txt", ours)
    finally:
        ctx.set_option(native.OPT_PARTICLE, 0)
    oracle_mod.set_electron(True)
    try:
        oracle_mod.bulk_run(d / "bulk.txt", theirs)
    finally:
        oracle_mod.set_electron(False)
    nnum, worst = compare(records(ours), records(theirs))
    assert nnum > 0 and worst <= 1e-9, worst
    ctx.set_option(native.OPT_RENORM_POLICY, 0)
    f2, _ = ctx.surf_run(theirs, d / "surf.txt", 0.1, 5, native.FP64)
    S = oracle_mod.Surface(theirs, d / "surf.txt", 0.1, 5)
    ref, _, _ = S.solve()
    S.close()
    abs_err, rel_err = spot_errors(f2, ref)
    assert abs_err <= 1e-10 and rel_err <= 1e-9, (abs_err, rel_err)
    # electrons and positrons scatter differently
    fp, _ = ctx.surf_run(d / "bulkP.b", d / "surf.txt", 0.1, 5, native.FP64)
    assert np.abs(fp - f2).max() > 1e-3 * np.abs(fp).max()
