"""Seeded synthetic structures written in the reference's input formats.

The reference reads two list-directed text files (format described in
str-orig/docs/html/_sources/index.rst.txt:219-330 and parsed by
sim-trhepd-rheed/src/bulkio.f90:34-113 and surfio.f90:125-195):

* ``bulk.txt``: beam set, energy and scan ranges, bulk cell and atoms;
* ``surf.txt``: surface elements, surface cell and atoms.

The reference never chooses beams itself; the generator's rule is: take the
``nbeam`` zero-order-Laue-zone rods with the smallest in-plane |G| on the
(1/nh, 1/nk) grid, ties broken by (ih, ik) ascending, with (0,0) first.

Workloads (sizes as published for the benchmark of this path):

* ``small23``  — N=23, square 3.84 A cell, 2-atom Si bulk, 3 Si surface layers,
  61 angles 0.5..6.5 deg, 15 A surface region, dz 0.02 A;
* ``batch47``  — N=47, 2x1 surface (7.68 x 3.84 A), 6 Si surface atoms,
  121 angles (0.05 deg) x 2 azimuths;
* ``dense521`` — N=521, 2x2 cell over a 4-atom bulk, 12 atoms Z in {14,32},
  61 angles, 20 A region, dz 0.01 A;
* ``uneven``   — 256 jittered candidates with N in {23,47,95,191};
* ``serving``  — Poisson request stream, N in {23,47,95,191,521}.
"""
from __future__ import annotations

import dataclasses
import math
from pathlib import Path

import numpy as np

A_SQ = 3.84      # square bulk lattice constant (A)
C_SQ = 3.14      # bulk layer spacing (A)


def _r6(x: float) -> float:
    """Values are held at the 6 decimals the text files carry."""
    return float(f"{x:.6f}")


@dataclasses.dataclass
class Element:
    z: int
    da1: float = 1.0     # valence correction of a(1) (bulkio.f90:73)
    sap: float = 0.15    # absorption ratio Im V / Re V (bulkio.f90:78)
    bh: float = 0.4
    bk: float = 0.4
    bz: float = 0.4

    def __post_init__(self):
        self.bh, self.bk, self.bz = _r6(self.bh), _r6(self.bk), _r6(self.bz)


@dataclasses.dataclass
class Atom:
    elem: int            # 1-based element index (surface file: >0 surface, <0 bulk)
    x: float
    y: float
    z: float
    occ: float = 1.0

    def __post_init__(self):
        self.x, self.y, self.z, self.occ = _r6(self.x), _r6(self.y), _r6(self.z), _r6(self.occ)


@dataclasses.dataclass
class Structure:
    """One bulk + surface pair ready to be written as bulk.txt / surf.txt."""
    nh: int
    nk: int
    beams: list[tuple[int, int]]
    energy_kev: float
    azi: tuple[float, float, float]           # start, end, step (deg)
    glancing: tuple[float, float, float]      # start, end, step (deg)
    bulk_dz: float
    ml: int
    bulk_elements: list[Element]
    nsg: int
    aa: float
    bb: float
    gam: float
    cc: float
    dx: float
    dy: float
    bulk_atoms: list[Atom]
    surf_elements: list[Element]
    nsgs: int
    msa: int
    msb: int
    nsa: int
    nsb: int
    dthick: float
    dxs: float
    dys: float
    surf_atoms: list[Atom]
    surface_dz: float = 0.02
    int_method: int = 5

    @property
    def nbeam(self) -> int:
        return len(self.beams)

    def bulk_text(self) -> str:
        ihik = ",".join(f"{h},{k}" for h, k in self.beams)
        L = [f"{self.nh},{self.nk},1\t\t\t,NH,NK,NDOM",
             f"{self.nbeam}\t\t\t,NB",
             "0\t\t\t,RDOM",
             f"{ihik}\t,(IH(I),IK(I)",
             "{:g},{:g},{:g},{:g},{:g},{:g},{:g}\t,BE,AZI,AZF,DAZ,GI,GF,DG".format(
                 self.energy_kev, *self.azi, *self.glancing),
             f"{self.bulk_dz:g},{self.ml}\t\t,DZ,ML",
             f"{len(self.bulk_elements)}\t\t\t,NELM"]
        for e in self.bulk_elements:
            L.append(f"{e.z},{e.da1:g},{e.sap:g}\t\t,Z,da1,sap")
            L.append(f"{e.bh:.6f},{e.bk:.6f},{e.bz:.6f}\t,BH(I),BK(I),BZ(I)")
        L.append(f"{self.nsg},{self.aa:.6f},{self.bb:.6f},{self.gam:g},{self.cc:.6f},"
                 f"{self.dx:.6f},{self.dy:.6f}\t,NSG,AA,BB,GAM,CC,DX,DY")
        L.append(f"{len(self.bulk_atoms)}\t\t\t,NATM")
        for a in self.bulk_atoms:
            L.append(f"{a.elem},{a.occ:.6f},{a.x:.6f},{a.y:.6f},{a.z:.6f}\t,IELM,ocr,X,Y,Z")
        return "\n".join(L) + "\n"

    def surf_text(self) -> str:
        L = [f"{len(self.surf_elements)}\t\t\t,NELMS"]
        for e in self.surf_elements:
            L.append(f"{e.z},{e.da1:g},{e.sap:g}\t\t,Z,da1,sap")
            L.append(f"{e.bh:.6f},{e.bk:.6f},{e.bz:.6f}\t,BH(I),BK(I),BZ(I)")
        L.append(f"{self.nsgs},{self.msa},{self.msb},{self.nsa},{self.nsb},{self.dthick:.6f},"
                 f"{self.dxs:.6f},{self.dys:.6f}\t,NSGS,msa,msb,nsa,nsb,dthick,DXS,DYS")
        L.append(f"{len(self.surf_atoms)}\t\t\t,NATM")
        for a in self.surf_atoms:
            L.append(f"{a.elem},{a.occ:.6f},{a.x:.6f},{a.y:.6f},{a.z:.6f}")
        return "\n".join(L) + "\n"

    def write(self, directory: str | Path) -> tuple[Path, Path]:
        d = Path(directory)
        d.mkdir(parents=True, exist_ok=True)
        (d / "bulk.txt").write_text(self.bulk_text())
        (d / "surf.txt").write_text(self.surf_text())
        return d / "bulk.txt", d / "surf.txt"


def zolz_beams(n: int, nh: int, nk: int, a: float, b: float) -> list[tuple[int, int]]:
    """The n rods with the smallest |G| on a square/rectangular (1/nh, 1/nk) grid."""
    gx, gy = 2 * math.pi / (a * nh), 2 * math.pi / (b * nk)
    r = int(math.ceil(math.sqrt(n))) + 4
    cand = []
    for h in range(-r * nh, r * nh + 1):
        for k in range(-r * nk, r * nk + 1):
            g2 = (gx * h) ** 2 + (gy * k) ** 2
            cand.append((round(g2, 9), h, k))
    cand.sort()
    out = [(h, k) for _, h, k in cand[:n]]
    assert out[0] == (0, 0)
    return out


def _bulk_square(rng: np.random.Generator, natm: int, b: float) -> list[Atom]:
    return [Atom(1, float(rng.uniform(0, 1)), float(rng.uniform(0, 1)),
                 float(rng.uniform(0, 1)) * C_SQ) for _ in range(natm)]


def _region_thickness(s: Structure, total: float) -> None:
    """Choose dthick so that the surface region (surfio.f90:201-205) spans `total` A."""
    zb = [a.z for a in s.bulk_atoms]
    zoffset = 0.5 * (s.cc - max(zb) - min(zb))
    zz = max(0.0, max(a.z for a in s.surf_atoms) + zoffset)
    s.dthick = _r6(max(0.5, total - s.cc - zz))


def small23(seed: int = 1) -> Structure:
    rng = np.random.default_rng(seed)
    bulk_atoms = _bulk_square(rng, 2, 0.4)
    ztop = max(a.z for a in bulk_atoms)
    surf = []
    for layer in range(3):
        h = float(rng.uniform(1.0, 6.0))
        for _ in range(2):
            surf.append(Atom(1, float(rng.uniform(0, 1)), float(rng.uniform(0, 1)), ztop + h))
    s = Structure(nh=1, nk=1, beams=zolz_beams(23, 1, 1, A_SQ, A_SQ), energy_kev=10.0,
                  azi=(0.0, 0.0, 0.0), glancing=(0.5, 6.5, 0.1), bulk_dz=0.05, ml=100,
                  bulk_elements=[Element(14, bh=0.4, bk=0.4, bz=0.4)], nsg=1, aa=A_SQ, bb=A_SQ,
                  gam=90.0, cc=C_SQ, dx=0.0, dy=0.0, bulk_atoms=bulk_atoms,
                  surf_elements=[Element(14, bh=0.8, bk=0.8, bz=0.8)], nsgs=1, msa=1, msb=0,
                  nsa=0, nsb=1, dthick=0.0, dxs=0.0, dys=0.0, surf_atoms=surf,
                  surface_dz=0.02, int_method=5)
    _region_thickness(s, 15.0)
    s.dthick = _r6(s.dthick)
    return s


def batch47(seed: int = 2) -> Structure:
    rng = np.random.default_rng(seed)
    bulk_atoms = _bulk_square(rng, 2, 0.4)
    ztop = max(a.z for a in bulk_atoms)
    elems, surf = [], []
    for layer in range(3):
        h = float(rng.uniform(1.0, 6.0))
        for _ in range(2):
            b = float(rng.uniform(0.3, 1.0))
            elems.append(Element(14, bh=b, bk=b, bz=b))
            surf.append(Atom(len(elems), float(rng.uniform(0, 2)), float(rng.uniform(0, 1)),
                             ztop + h))
    s = Structure(nh=2, nk=1, beams=zolz_beams(47, 2, 1, A_SQ, A_SQ), energy_kev=10.0,
                  azi=(0.0, 90.0, 90.0), glancing=(0.5, 6.5, 0.05), bulk_dz=0.05, ml=100,
                  bulk_elements=[Element(14)], nsg=1, aa=A_SQ, bb=A_SQ, gam=90.0, cc=C_SQ,
                  dx=0.0, dy=0.0, bulk_atoms=bulk_atoms, surf_elements=elems, nsgs=1, msa=2,
                  msb=0, nsa=0, nsb=1, dthick=0.0, dxs=0.0, dys=0.0, surf_atoms=surf,
                  surface_dz=0.02, int_method=5)
    _region_thickness(s, 15.0)
    return s


def dense(n: int = 521, seed: int = 3, n_angles: int = 61, region: float = 20.0,
          dz: float = 0.01) -> Structure:
    """2x2 reconstructed cell over a 4-atom bulk, surface atoms Z in {14, 32}."""
    rng = np.random.default_rng(seed)
    bulk_atoms = _bulk_square(rng, 4, 0.4)
    ztop = max(a.z for a in bulk_atoms)
    elems, surf = [], []
    layers = np.sort(rng.uniform(0.0, 8.0, size=4))
    for i in range(12):
        z = int(rng.choice([14, 32]))
        b = float(rng.uniform(0.3, 1.2))
        elems.append(Element(z, bh=b, bk=b, bz=b))
        surf.append(Atom(len(elems), float(rng.uniform(0, 2)), float(rng.uniform(0, 2)),
                         ztop + 0.5 + float(layers[i % 4])))
    step = 6.0 / (n_angles - 1) if n_angles > 1 else 0.0
    s = Structure(nh=2, nk=2, beams=zolz_beams(n, 2, 2, A_SQ, A_SQ), energy_kev=10.0,
                  azi=(0.0, 0.0, 0.0), glancing=(0.5, 0.5 + step * (n_angles - 1), step),
                  bulk_dz=0.05, ml=100, bulk_elements=[Element(14)], nsg=1, aa=A_SQ, bb=A_SQ,
                  gam=90.0, cc=C_SQ, dx=0.0, dy=0.0, bulk_atoms=bulk_atoms, surf_elements=elems,
                  nsgs=1, msa=2, msb=0, nsa=0, nsb=2, dthick=0.0, dxs=0.0, dys=0.0,
                  surf_atoms=surf, surface_dz=dz, int_method=5)
    _region_thickness(s, region)
    return s


def dense521(seed: int = 3) -> Structure:
    return dense(521, seed)


def jitter(base: Structure, sigma: float, seed: int) -> Structure:
    """A candidate surface: the base structure with surface atoms moved by N(0, sigma) A."""
    rng = np.random.default_rng(seed)
    s = dataclasses.replace(base)
    s.surf_atoms = [dataclasses.replace(
        a, x=a.x + float(rng.normal(0, sigma)) / (s.aa),
        y=a.y + float(rng.normal(0, sigma)) / (s.bb),
        z=a.z + float(rng.normal(0, sigma))) for a in base.surf_atoms]
    return s


WORKLOADS = {"small23": small23, "batch47": batch47, "dense521": dense521}
