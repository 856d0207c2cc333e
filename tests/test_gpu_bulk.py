"""GPU bulk solve (trhepd_bulk_run: bulk.txt -> bulkP.b) against the reference.

The reference's bulkP.b files (tests/golden/*/bulkP.b, written by the original
eigen-decomposition path of trmat, sim-trhepd-rheed/src/bulk.f90:130-264) pin the
reflection records; the GPU builds the slice transfer matrix from the matrix
cosine/sine series instead of eigenvectors, so records agree to rounding of
the two constructions.  Header records must be byte-identical.  Synthetic
structures are checked against the oracle's restatement.
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


@pytest.mark.parametrize("n,seed", [(23, 5), (95, 7)])
def test_bulk_synthetic_vs_oracle(oracle_mod, ctx, tmp_path, n, seed):
    from trhepd_opt_b200 import generator
    s = generator.dense(n, seed=seed, n_angles=7, region=4.0, dz=0.02)
    bulk_txt, _ = s.write(tmp_path)
    ours, theirs = tmp_path / "gpu.b", tmp_path / "oracle.b"
    ctx.bulk_run(bulk_txt, ours)
    oracle_mod.bulk_run(bulk_txt, theirs)
    nnum, worst = compare(records(ours), records(theirs))
    assert nnum > 0
    assert worst <= 1e-8, worst


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
