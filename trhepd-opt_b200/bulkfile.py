"""bulkP.b writer: the header half of the reference's bulk program.

Restates bulkio's output records (sim-trhepd-rheed/src/bulkio.f90:126-141 and
:173-176) with the beam grouping of blkibg (bulksub.f90:46-92) and the
beam-difference list of blkghk (bulksub.f90:96-135), as Fortran unformatted
sequential records (4-byte length markers).

The per-(angle, group) reflection records that follow (bulk.f90:122) come from
a callable ``records(angle_index, group_index, nbf) -> complex (nbf, nbf)``
(column-major as written by the reference).  ``zero_records`` writes a
non-reflecting bulk (f = 0); the surface solve's cost does not depend on the
record values.
"""
from __future__ import annotations

import math
import struct
from pathlib import Path

import numpy as np

from .generator import Structure
from . import scattering

RAD = math.pi / 180.0


def _rec(f, payload: bytes) -> None:
    n = struct.pack("<i", len(payload))
    f.write(n + payload + n)


def blkibg(nb: int, ih: list[int], ik: list[int], nh: int, nk: int):
    """Beam groups coupled in the bulk; reorders ih/ik in place (bulksub.f90:46-92)."""
    iord = list(range(1, nb + 1))
    if nh == 1 and nk == 1:
        return iord, [nb]
    nbg = []
    j = 1
    while True:
        i = j
        j = i + 1
        ih0, ik0 = ih[i - 1], ik[i - 1]
        for k in range(i + 1, nb + 1):
            if (ih[k - 1] - ih0) % nh == 0 and (ik[k - 1] - ik0) % nk == 0:
                if k > j:
                    l, n, m = ih[k - 1], ik[k - 1], iord[k - 1]
                    for jj in range(k, j, -1):
                        ih[jj - 1], ik[jj - 1], iord[jj - 1] = ih[jj - 2], ik[jj - 2], iord[jj - 2]
                    ih[j - 1], ik[j - 1], iord[j - 1] = l, n, m
                j += 1
        nbg.append(j - i)
        if j > nb:
            return iord, nbg


def blkghk(nbg: list[int], ih: list[int], ik: list[int]):
    """Distinct in-group beam differences, (0,0) first (bulksub.f90:96-135)."""
    igh, igk = [0], [0]
    index = {}
    ibas = 0
    for g in nbg:
        iend = ibas + g
        for k in range(ibas, iend - 1):
            for l in range(k + 1, iend):
                key = (ih[l] - ih[k], ik[l] - ik[k])
                if key not in index:
                    index[key] = len(igh)
                    igh.append(key[0])
                    igk.append(key[1])
        ibas = iend
    return igh, igk


def scan_count(start: float, end: float, step: float) -> int:
    """naz / ng of scanrg (bulksub.f90:9-42)."""
    if abs(step) < 1e-4:
        return 1
    return min(max(int((end - start) / step + 0.1) + 1, 1), 200)


def zero_records(angle: int, group: int, nbf: int) -> np.ndarray:
    return np.zeros((nbf, nbf), dtype=np.complex128)


def write_bulkp(s: Structure, path, records=zero_records, electron: bool = False) -> dict:
    """Write bulkP.b for structure `s` (one domain; positrons, or electrons with
    inegpos = 0 and no sign flip, bulkm.f90:21-24); returns header data."""
    ih = [h for h, _ in s.beams]
    ik = [k for _, k in s.beams]
    nb = len(ih)
    elems = s.bulk_elements
    zb = [a.z for a in s.bulk_atoms]
    zoffset = 0.5 * (s.cc - max(zb) - min(zb))
    naz = scan_count(*s.azi)
    ng = scan_count(*s.glancing)
    ns = int(s.cc / s.bulk_dz) + 1
    dz = s.cc / ns
    ml = s.ml if 1 <= s.ml <= 1000 else 1000
    nabr, nabi = 4, 1
    with open(path, "wb") as f:
        _rec(f, struct.pack("<i", 1))
        _rec(f, struct.pack("<10i", 0 if electron else 1, 0, s.nh, s.nk, 0, 1, 0, nabr, nabi, 3))
        _rec(f, struct.pack("<id", nb, 0.0))
        _rec(f, b"".join(struct.pack("<ii", h, k) for h, k in zip(ih, ik)))
        _rec(f, struct.pack("<dddiddi", s.energy_kev, s.azi[0] * RAD, s.azi[2] * RAD, naz,
                            s.glancing[0] * RAD, s.glancing[2] * RAD, ng))
        _rec(f, struct.pack("<ddid", 0.0, dz, ml, 1e-10))
        _rec(f, struct.pack("<ii7d", s.nsg, 0, s.aa, s.bb, s.gam * RAD, s.cc, s.dx, s.dy,
                            zoffset))
        _rec(f, struct.pack("<ii", len(elems), len(s.bulk_atoms)))
        for e in elems:
            a, b = scattering.params(e.z)
            a = list(a)
            a[0] -= e.da1
            if not electron:
                a = [-x for x in a]  # positron (bulkio.f90:74)
            _rec(f, struct.pack("<10d", *a, e.sap, *b, 0.0))
            _rec(f, struct.pack("<5d", e.bh, e.bk, e.bz, scattering.mass(e.z), 0.0))
        for at in s.bulk_atoms:
            _rec(f, struct.pack("<i4d", at.elem, at.occ, at.x, at.y, at.z + zoffset))
        ihs, iks = list(ih), list(ik)
        iord, nbg = blkibg(nb, ihs, iks, s.nh, s.nk)
        igh, igk = blkghk(nbg, ihs, iks)
        _rec(f, struct.pack(f"<{nb}i", *iord))
        _rec(f, struct.pack("<ii", len(nbg), len(igh)))
        _rec(f, struct.pack(f"<{len(nbg)}i", *nbg))
        _rec(f, b"".join(struct.pack("<ii", h, k) for h, k in zip(igh, igk)))
        nrep = naz * ng
        for t in range(nrep):
            for gi, g in enumerate(nbg):
                m = np.asarray(records(t, gi, g), dtype=np.complex128)
                _rec(f, np.asfortranarray(m).tobytes(order="F"))
    return {"nb": nb, "naz": naz, "ng": ng, "nbg": nbg, "iord": iord, "nvb": len(igh)}
