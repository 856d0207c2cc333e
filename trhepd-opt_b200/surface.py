"""Python mirror of the reference's surface-solve interface.

``SurfaceProblem`` plays surfio (sim-trhepd-rheed/src/surfio.f90:60-381): it
reads the unchanged bulkP.b / surf.txt and exposes the mod_scpot3 state and
srfref's arguments.  ``srfref`` calls the C-ABI replacement of srfref
(surflf.f90:7-171) and ``potential_table`` the replacement of the integrator
init routines (surf_prkn.f90:174-197).  Everything runs through the CUDA
library; there is no CPU path.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import native


class SurfaceProblem:
    def __init__(self, ctx: native.Context, bulkp, surf, dz2: float, int_method: int = 5):
        h = ctypes.c_void_p()
        L = native.load()
        ctx._check(L.trhepd_surf_load(ctx._h, str(bulkp).encode(), str(surf).encode(),
                                      float(dz2), int(int_method), ctypes.byref(h)))
        self._h, self._L, self.ctx = h, L, ctx
        self.pot = native.PotState()
        self.args = native.SrfrefArgs()
        ctx._check(L.trhepd_surf_views(h, ctypes.byref(self.pot), ctypes.byref(self.args)))

    @property
    def n_angles(self) -> int:
        return self.args.nrep1 * self.args.nrep2

    def srfref(self, precision: int = native.FP64):
        """All (azimuth, angle) solves of the domain: (angles_deg, f2[nangles, nb])."""
        a = self.args
        f2 = np.zeros((self.n_angles, a.nb))
        ang = np.zeros(self.n_angles)
        self.ctx._check(self._L.trhepd_srfref(
            self.ctx._h, ctypes.byref(self.pot), a.nb, a.ns, a.iv, a.dz, a.ngr, a.nbg, a.iord,
            a.ih, a.ik, a.wn, a.ghx, a.ghy, a.gky, a.azi, a.daz, a.naz, a.gi, a.dg, a.ng,
            a.int_method, a.t1_records, int(precision), f2.ctypes.data, ang.ctypes.data))
        return ang, f2

    def potential_table(self, int_method: int | None = None):
        """Stage potential tables v, vi as (ncol, nv) complex arrays."""
        m = self.args.int_method if int_method is None else int_method
        ncol = table_columns(m, self.args.ns)
        v = np.zeros((ncol, self.pot.nv), dtype=np.complex128)
        vi = np.zeros_like(v)
        nc = ctypes.c_int(0)
        self.ctx._check(self._L.trhepd_potential_table(
            self.ctx._h, ctypes.byref(self.pot), m, self.args.ns, self.args.dz,
            v.ctypes.data, vi.ctypes.data, ctypes.byref(nc)))
        assert nc.value == ncol
        return v, vi

    def resident(self) -> "ResidentProblem":
        """Upload this problem and build its stage tables in device memory."""
        return ResidentProblem(self)

    def close(self):
        if getattr(self, "_h", None):
            self._L.trhepd_surf_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def table_columns(int_method: int, ns: int) -> int:
    """Stage-table columns of each integrator's init routine (surf_prkn.f90:174-197,
    surf_magnus.f90:4-42, surf_rk.f90:4-25)."""
    per = {1: (1, 0), 2: (3, 0), 3: (3, 0), 4: (1, 0), 5: (6, 1), 6: (11, 1), 7: (2, 1)}
    if int_method not in per:
        raise ValueError("the GPU path integrates int_method 1 to 7")
    s, extra = per[int_method]
    return s * ns + extra


def potential_table(ctx: native.Context, bulkp, surf, dz2: float, int_method: int = 5):
    return SurfaceProblem(ctx, bulkp, surf, dz2, int_method).potential_table()


def srfref(ctx: native.Context, bulkp, surf, dz2: float, int_method: int = 5,
           precision: int = native.FP64):
    return SurfaceProblem(ctx, bulkp, surf, dz2, int_method).srfref(precision)


class ResidentProblem:
    """A srfref problem held in device memory (trhepd_problem_*)."""

    def __init__(self, sp: SurfaceProblem):
        self.sp, self.ctx, self._L = sp, sp.ctx, sp._L
        h = ctypes.c_void_p()
        self.ctx._check(self._L.trhepd_problem_create(self.ctx._h, ctypes.byref(sp.pot),
                                                      ctypes.byref(sp.args), ctypes.byref(h)))
        self._h = h
        info = np.zeros(6, dtype=np.int64)
        self._L.trhepd_problem_info(h, info.ctypes.data, 6)
        self.nb, self.nangles, self.ns, self.nv, self.ncol, self.device_bytes = map(int, info)

    def solve(self, precision: int = native.FP64):
        """Integrate every angle; the intensities stay on the device."""
        self.ctx._check(self._L.trhepd_problem_solve(self.ctx._h, self._h, int(precision)))

    def fetch(self):
        f2 = np.zeros((self.nangles, self.nb))
        ang = np.zeros(self.nangles)
        self.ctx._check(self._L.trhepd_problem_fetch(self.ctx._h, self._h, f2.ctypes.data,
                                                     ang.ctypes.data))
        return ang, f2

    def compare(self, ref_f2):
        """compare.py's per-angle metric between the solved curves and `ref_f2`
        (nangles, nb), reduced on the device: (nangles, 2) = (e0 / max n0, e0 / n0)."""
        ref = np.ascontiguousarray(ref_f2, dtype=np.float64)
        if ref.shape != (self.nangles, self.nb):
            raise ValueError(f"reference curves must be {(self.nangles, self.nb)}")
        out = np.zeros((self.nangles, 2))
        self.ctx._check(self._L.trhepd_problem_compare(self.ctx._h, self._h, ref.ctypes.data,
                                                       out.ctypes.data))
        return out

    def convolve(self, omega: float = 0.5):
        """The solved intensities convolved on the device (make_convolution.py)."""
        out = np.zeros((self.nangles, self.nb))
        self.ctx._check(self._L.trhepd_problem_convolve(self.ctx._h, self._h, float(omega),
                                                        out.ctypes.data))
        return out

    def close(self):
        if getattr(self, "_h", None):
            self._L.trhepd_problem_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_batch(ctx: native.Context, problems, precision: int = native.FP64) -> None:
    """Solve resident problems together (trhepd_batch_solve): the small-beam RKN
    ones share fused launches whatever their beam counts and angle grids, the
    others run one after another; read each with its fetch()."""
    problems = list(problems)
    arr = (ctypes.c_void_p * len(problems))(*[p._h.value for p in problems])
    ctx._check(ctx._L.trhepd_batch_solve(ctx._h, arr, len(problems), int(precision)))

