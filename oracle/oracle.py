"""CPU oracle loader — test infrastructure, not the product.

ctypes front-end for ``oracle/_build/liboracle.so``, the FP64 C++ restatement
of the sim-trhepd-rheed surface and bulk solves.  Only ``tests/``, the smoke
check and ``bench.py``'s CPU-baseline leg may import this module; the product
path never does.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"
_lib = None


def build(quiet: bool = True) -> Path:
    """Compile the oracle with its Makefile (g++ -fopenmp, scipy's OpenBLAS)."""
    cmd = ["make", "-C", str(HERE)]
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        L.oracle_surface_open.restype = ctypes.c_void_p
        L.oracle_surface_open.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_double,
                                          ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        L.oracle_surface_close.argtypes = [ctypes.c_void_p]
        L.oracle_surface_dims.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
        L.oracle_surface_scalars.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        L.oracle_surface_tables.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_void_p]
        L.oracle_surface_solve.restype = ctypes.c_int
        L.oracle_surface_solve.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_surface_solve_list.restype = ctypes.c_int
        L.oracle_surface_solve_list.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_surface_kappa_max.restype = ctypes.c_double
        L.oracle_surface_kappa_max.argtypes = [ctypes.c_void_p]
        L.oracle_set_renorm_every.argtypes = [ctypes.c_int]
        L.oracle_surface_write.restype = ctypes.c_int
        L.oracle_surface_write.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.oracle_bulk_run.restype = ctypes.c_int
        L.oracle_bulk_run.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                      ctypes.c_int]
        L.oracle_set_threads.argtypes = [ctypes.c_int]
        L.oracle_set_max_slices.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def set_threads(n: int | None = None) -> int:
    n = n or os.cpu_count() or 1
    lib().oracle_set_threads(int(n))
    return n


class Surface:
    """One surf.exe problem (bulkP.b + surf.txt + dz2 + int_method), domain 1."""

    def __init__(self, bulkp: str | os.PathLike, surf: str | os.PathLike, dz2: float,
                 method: int = 5):
        err = ctypes.create_string_buffer(512)
        h = lib().oracle_surface_open(str(bulkp).encode(), str(surf).encode(), float(dz2),
                                      int(method), err, 512)
        if not h:
            raise RuntimeError("oracle: " + err.value.decode())
        self._h = h
        d = (ctypes.c_int * 10)()
        lib().oracle_surface_dims(h, d)
        (self.nb, self.nv, self.nvb, self.ns, self.ncol, self.nrep1, self.nrep2, self.ngr,
         self.naz, self.ng) = list(d)
        s = (ctypes.c_double * 9)()
        lib().oracle_surface_scalars(h, s)
        self.dz, self.wn, self.ghx, self.ghy, self.gky, self.azi, self.daz, self.gi, self.dg = list(s)
        self.method = method

    @property
    def n_angles(self) -> int:
        return self.nrep1 * self.nrep2

    def tables(self):
        v = np.empty((self.ncol, self.nv), dtype=np.complex128)
        vi = np.empty((self.ncol, self.nv), dtype=np.complex128)
        iv = np.empty((self.nb, self.nb), dtype=np.int32)
        lib().oracle_surface_tables(self._h, v.ctypes.data, vi.ctypes.data, iv.ctypes.data)
        return v, vi, iv  # v[c, k] = column c; iv[j, i] = Fortran iv(i+1, j+1)

    def solve(self, first: int = 0, count: int | None = None):
        count = self.n_angles - first if count is None else count
        f2 = np.empty((count, self.nb), dtype=np.float64)
        ang = np.empty(count, dtype=np.float64)
        ren = np.empty(count, dtype=np.int32)
        rc = lib().oracle_surface_solve(self._h, first, count, f2.ctypes.data, ang.ctypes.data,
                                        ren.ctypes.data)
        if rc:
            raise RuntimeError(f"oracle solve failed rc={rc}")
        return f2, ang, ren

    def solve_list(self, idx):
        """Solve the listed angles (schedule indices) in parallel, one per thread."""
        idx = np.ascontiguousarray(idx, dtype=np.int32)
        f2 = np.empty((len(idx), self.nb), dtype=np.float64)
        ang = np.empty(len(idx), dtype=np.float64)
        ren = np.empty(len(idx), dtype=np.int32)
        rc = lib().oracle_surface_solve_list(self._h, idx.ctypes.data, len(idx), f2.ctypes.data,
                                             ang.ctypes.data, ren.ctypes.data)
        if rc:
            raise RuntimeError(f"oracle solve failed rc={rc}")
        return f2, ang, ren

    def kappa_max(self) -> float:
        """Largest evanescent decay constant over the beams and angles of the scan."""
        return float(lib().oracle_surface_kappa_max(self._h))

    def write(self, path) -> None:
        rc = lib().oracle_surface_write(self._h, str(path).encode())
        if rc:
            raise RuntimeError(f"oracle write failed rc={rc}")

    def close(self):
        if self._h:
            lib().oracle_surface_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bulk_run(bulk_txt, out_path) -> None:
    err = ctypes.create_string_buffer(512)
    rc = lib().oracle_bulk_run(str(bulk_txt).encode(), str(out_path).encode(), err, 512)
    if rc:
        raise RuntimeError("oracle bulk: " + err.value.decode())


def set_bulk_scale(s: float) -> None:
    """Rescale the bulk slice potentials by s in bulk_run (1 = off); a scale of
    1 + 2^-50 measures the rounding sensitivity of each bulk record."""
    lib().oracle_set_bulk_scale(ctypes.c_double(s))


def set_electron(on: bool) -> None:
    """bulk_run for electrons (inegpos = 0, bulkm.f90:21-24) or positrons (default)."""
    lib().oracle_set_electron(1 if on else 0)


def set_renorm_every(k: int) -> None:
    """0: the reference's Gershgorin renormalisation test (default); k > 0:
    renormalise after every k-th slice instead (a growth-bound schedule)."""
    lib().oracle_set_renorm_every(int(k))


def growth_interval(kappa_max: float, dz: float, tau: float = math.log(1e3)) -> int:
    """Slices between renormalisations of the growth-bound schedule: the largest
    L with exp((kappa_max + 1) L dz) <= exp(tau)."""
    return max(1, int(math.floor(tau / ((kappa_max + 1.0) * dz))))


def set_max_slices(n: int) -> None:
    """Integrate only the first n slices (0 = all); for bounded timing samples."""
    lib().oracle_set_max_slices(int(n))


def rocking_convolution(angle_deg, f2, omega: float = 0.5, scan: int | None = None):
    """Gaussian convolution of rocking curves along the scanned angle, restating
    the reference's make_convolution.py (str-lapack/tool/make_convolution.py:21-29
    for sigma = omega / (2 sqrt(2 ln 2)) and the normalised Gaussian, :97-109 for
    C_i = sum_k I_k g(theta_i - theta_k) dtheta with dtheta = theta_1 - theta_0).
    Rows come in consecutive blocks of `scan` angles (one block per outer loop
    index of srfref; the script handles one block); each block is convolved alone."""
    import numpy as np
    angle_deg = np.asarray(angle_deg, dtype=float)
    f2 = np.asarray(f2, dtype=float)
    scan = scan or len(angle_deg)
    sigma = 0.5 * omega / np.sqrt(2.0 * np.log(2.0))
    out = np.zeros_like(f2)
    for b0 in range(0, len(angle_deg), scan):
        a = angle_deg[b0:b0 + scan]
        d = a[1] - a[0]
        x = a[:, None] - a[None, :]
        g = (1.0 / (sigma * np.sqrt(2.0 * np.pi))) * np.exp(-0.5 * x ** 2 / sigma ** 2)
        out[b0:b0 + scan] = (g * d) @ f2[b0:b0 + scan]
    return out


def compare_curves(comp, ref):
    """The per-angle metric of the reference's regression scripts, restating
    test/test23/compare.py:50-67: for each angle row, n0 = ||comp||_2 (1 when 0) and
    e0 = ||comp - ref||_2; returns (nangles, 2) = (e0 / max_a n0, e0 / n0), the two
    numbers the script prints after the angle."""
    comp = np.asarray(comp, dtype=float)
    ref = np.asarray(ref, dtype=float)
    n0 = np.linalg.norm(comp, axis=1)
    n0 = np.where(n0 == 0.0, 1.0, n0)
    e0 = np.linalg.norm(comp - ref, axis=1)
    return np.stack([e0 / n0.max(), e0 / n0], axis=1)


def _fortran_e_value(v: float, d: int) -> float:
    """v as Fortran's E(w).d edit writes it (d significant digits, 0.ddd form) and
    reads it back."""
    if v == 0.0:
        return 0.0
    m, e = f"{abs(v):.{d - 1}e}".split("e")
    digits = m.replace(".", "")
    return float(("-" if v < 0 else "") + "0." + digits + "e" + str(int(e) + 1))


def domain_curves(S: "Surface"):
    """Every domain of a multi-domain problem solved by the oracle: list of
    (angle_deg, f2[nangles, nb_d]) in domain order (surfio.f90:291-341)."""
    L = lib()
    L.oracle_surface_solve_domain.restype = ctypes.c_int
    L.oracle_surface_solve_domain.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    hdr = domain_header(S)
    out = []
    for d, nb in enumerate(hdr["nbd"]):
        f2 = np.empty((S.n_angles, nb))
        ang = np.empty(S.n_angles)
        if L.oracle_surface_solve_domain(S._h, d, 0, S.n_angles, f2.ctypes.data, ang.ctypes.data):
            raise RuntimeError("oracle domain solve failed")
        out.append((ang, f2))
    return out


def domain_header(S: "Surface") -> dict:
    """nbd, rdom (rad), wdom, gam (rad), every domain's ih/ik, nh, nk of a problem."""
    L = lib()
    L.oracle_surface_domains.argtypes = [ctypes.c_void_p] * 8
    nhnk = (ctypes.c_int * 3)()
    L.oracle_surface_domains(S._h, None, None, None, None, None, None, nhnk)
    ndom = nhnk[2]
    nbd = np.zeros(ndom, dtype=np.int32)
    rdom, wdom = np.zeros(ndom), np.zeros(ndom)
    gam = ctypes.c_double()
    L.oracle_surface_domains(S._h, nbd.ctypes.data, rdom.ctypes.data, wdom.ctypes.data,
                             ctypes.byref(gam), None, None, nhnk)
    ih = np.zeros(int(nbd.sum()), dtype=np.int32)
    ik = np.zeros_like(ih)
    L.oracle_surface_domains(S._h, None, None, None, None, ih.ctypes.data, ik.ctypes.data, nhnk)
    return {"nbd": [int(x) for x in nbd], "rdom": rdom, "wdom": wdom, "gam": gam.value,
            "ih": ih, "ik": ik, "nh": nhnk[0], "nk": nhnk[1]}


def domain_sum(curves, hdr):
    """Weighted sum of rotated-domain rocking curves, restating
    sim-trhepd-rheed/src/domainsum.f90:7-121 on values as it reads them from the .md
    header (domain angles and cell angle F10.3 degrees, weights E12.3): the reference
    domain has the most beams (first such); a beam of another domain is added onto
    the first reference beam within 1e-4 after rotation by rdom(ref) - rdom(d)
    (reduced coordinates h/nh, k/nk, sheared for gam = 120 deg), sums in domain and
    beam order.  Returns (angle_deg of the last domain, s2[nangles, mb], idomr)."""
    rad = math.atan(1.0) / 45.0
    deg = 1.0 / rad
    nbd = hdr["nbd"]
    ndom = len(nbd)
    gam = float(f"{hdr['gam'] * deg:10.3f}")
    rdom = [float(f"{r * deg:10.3f}") for r in hdr["rdom"]]
    wdom = [_fortran_e_value(w, 3) for w in hdr["wdom"]]
    idomr = int(np.argmax(nbd))
    mb = nbd[idomr]
    off = np.concatenate([[0], np.cumsum(nbd)])

    def red(b):
        gx, gy = hdr["ih"][b] / hdr["nh"], hdr["ik"][b] / hdr["nk"]
        if abs(gam - 120.0) < 1e-4:
            gx = (gx + gx + gy) / math.sqrt(3.0)
        return gx, gy

    nang = curves[0][1].shape[0]
    s2 = np.zeros((nang, mb))
    for d in range(ndom):
        f2 = curves[d][1]
        if d == idomr:
            for ib in range(mb):
                s2[:, ib] = s2[:, ib] + f2[:, ib] * wdom[d]
            continue
        dr = rdom[idomr] - rdom[d]
        cdr, sdr = math.cos(dr * rad), math.sin(dr * rad)
        for ib in range(nbd[d]):
            gx, gy = red(off[d] + ib)
            gxr, gyr = cdr * gx - sdr * gy, sdr * gx + cdr * gy
            for ibr in range(mb):
                hx, hy = red(off[idomr] + ibr)
                if abs(gxr - hx) < 1e-4 and abs(gyr - hy) < 1e-4:
                    s2[:, ibr] = s2[:, ibr] + f2[:, ib] * wdom[d]
                    break
    return curves[-1][0], s2, idomr
