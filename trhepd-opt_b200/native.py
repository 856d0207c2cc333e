"""ctypes binding of the sm_100a library (include/trhepd_b200.h).

The library is built in-tree by ``build.py``.  There is no CPU fallback: if
the shared library is missing or no CUDA device is visible, every entry point
raises ``NativeUnavailable``.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_lib" / "libtrhepd_b200.so"

FP64 = 0
SPLIT_BF16 = 1
SPLIT_INT8 = 2
OPT_RENORM_POLICY = 1
OPT_RENORM_TAU = 2
OPT_SPLIT_SLICES = 3
OPT_PROFILE = 4
OPT_SPLIT_KERNEL = 5
OPT_GRAPHS = 6
OPT_FUSED_MAX_N = 7
OPT_STREAM_PRIORITY = 8
OPT_VALIDATE = 9
OPT_PARTICLE = 10
OPT_MAX_CTAS = 11

# every symbol include/trhepd_b200.h declares
EXPORTS = [
    "trhepd_create", "trhepd_destroy", "trhepd_last_error", "trhepd_set_option",
    "trhepd_last_stats", "trhepd_structure_factors", "trhepd_plane_group_images",
    "trhepd_potential_table", "trhepd_srfref", "trhepd_surf_run", "trhepd_surf_load",
    "trhepd_surf_free", "trhepd_surf_views", "trhepd_problem_create", "trhepd_problem_solve", "trhepd_batch_solve", "trhepd_rocking_convolution", "trhepd_problem_convolve",
    "trhepd_problem_fetch", "trhepd_problem_info", "trhepd_problem_destroy",
    "trhepd_potential_table_noalloc", "trhepd_bulk_run", "trhepd_last_curve_errors",
    "trhepd_problem_compare",
]


class PotState(ctypes.Structure):
    """trhepd_pot_state (mirrors mod_scpot3, surfio.f90:18-27)."""
    _fields_ = [("nv", ctypes.c_int), ("nvb", ctypes.c_int), ("natms", ctypes.c_int),
                ("natmb", ctypes.c_int), ("nelm", ctypes.c_int), ("nabr", ctypes.c_int),
                ("nabi", ctypes.c_int), ("ielm", ctypes.c_void_p), ("cc", ctypes.c_double),
                ("smesh", ctypes.c_double), ("z", ctypes.c_void_p), ("dchg", ctypes.c_void_p),
                ("Ghk", ctypes.c_void_p), ("ocr", ctypes.c_void_p), ("b", ctypes.c_void_p),
                ("asf", ctypes.c_void_p), ("st0", ctypes.c_void_p), ("st1", ctypes.c_void_p),
                ("st2", ctypes.c_void_p)]


class SrfrefArgs(ctypes.Structure):
    """trhepd_srfref_args: srfref's arguments (surflf.f90:7-8)."""
    _fields_ = [("nb", ctypes.c_int), ("ns", ctypes.c_int), ("iv", ctypes.c_void_p),
                ("dz", ctypes.c_double), ("ngr", ctypes.c_int), ("nbg", ctypes.c_void_p),
                ("iord", ctypes.c_void_p), ("ih", ctypes.c_void_p), ("ik", ctypes.c_void_p),
                ("wn", ctypes.c_double), ("ghx", ctypes.c_double), ("ghy", ctypes.c_double),
                ("gky", ctypes.c_double), ("azi", ctypes.c_double), ("daz", ctypes.c_double),
                ("naz", ctypes.c_int), ("gi", ctypes.c_double), ("dg", ctypes.c_double),
                ("ng", ctypes.c_int), ("int_method", ctypes.c_int),
                ("t1_records", ctypes.c_void_p), ("nrep1", ctypes.c_int),
                ("nrep2", ctypes.c_int)]

STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "non-finite / zero pivot",
          4: "device wait timed out", 5: "out of memory / over budget", 6: "input file error"}


class NativeUnavailable(RuntimeError):
    pass


class TrhepdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"trhepd status {code} ({STATUS.get(code, '?')}): {msg}")
        self.code = code


_lib = None
_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double


def load():
    """Load the shared library (raises NativeUnavailable if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        raise NativeUnavailable(f"{LIB} is not built (run trhepd-opt_b200/build.py)")
    L = ctypes.CDLL(str(LIB))
    L.trhepd_create.argtypes = [_I, ctypes.POINTER(_P)]
    L.trhepd_destroy.argtypes = [_P]
    L.trhepd_destroy.restype = None
    L.trhepd_last_error.argtypes = [_P]
    L.trhepd_last_error.restype = ctypes.c_char_p
    L.trhepd_set_option.argtypes = [_P, _I, _D]
    L.trhepd_last_stats.argtypes = [_P, _P, _I]
    L.trhepd_structure_factors.argtypes = [_P, _I, _P, _P, _I, _P, _P, _D, _D, _P]
    L.trhepd_plane_group_images.argtypes = [_I, _I, _I, _I, _I, _D, _D, _P, _P]
    L.trhepd_potential_table.argtypes = [_P, _P, _I, _I, _D, _P, _P, _P]
    L.trhepd_srfref.argtypes = [_P, _P, _I, _I, _P, _D, _I, _P, _P, _P, _P, _D, _D, _D, _D,
                                _D, _D, _I, _D, _D, _I, _I, _P, _I, _P, _P]
    L.trhepd_surf_run.argtypes = [_P, ctypes.c_char_p, ctypes.c_char_p, _D, _I, _I,
                                  ctypes.c_char_p, _P, _I, _P]
    L.trhepd_surf_load.argtypes = [_P, ctypes.c_char_p, ctypes.c_char_p, _D, _I,
                                   ctypes.POINTER(_P)]
    L.trhepd_surf_free.argtypes = [_P]
    L.trhepd_surf_free.restype = None
    L.trhepd_surf_views.argtypes = [_P, ctypes.POINTER(PotState), ctypes.POINTER(SrfrefArgs)]
    L.trhepd_problem_create.argtypes = [_P, ctypes.POINTER(PotState), ctypes.POINTER(SrfrefArgs),
                                        ctypes.POINTER(_P)]
    L.trhepd_problem_solve.argtypes = [_P, _P, _I]
    L.trhepd_batch_solve.argtypes = [_P, _P, _I, _I]
    L.trhepd_rocking_convolution.argtypes = [_P, _P, _P, _I, _I, _I, _D, _P]
    L.trhepd_problem_convolve.argtypes = [_P, _P, _D, _P]
    L.trhepd_problem_fetch.argtypes = [_P, _P, _P, _P]
    L.trhepd_last_curve_errors.argtypes = [_P, _P, _I]
    L.trhepd_problem_compare.argtypes = [_P, _P, _P, _P]
    L.trhepd_problem_info.argtypes = [_P, _P, _I]
    L.trhepd_potential_table_noalloc.argtypes = [_P, _I, _I, _D, _P, _P, _P]
    L.trhepd_bulk_run.argtypes = [_P, ctypes.c_char_p, ctypes.c_char_p, _P]
    L.trhepd_problem_destroy.argtypes = [_P]
    L.trhepd_problem_destroy.restype = None
    for name in EXPORTS:
        if name not in ("trhepd_destroy", "trhepd_last_error", "trhepd_surf_free",
                        "trhepd_problem_destroy"):
            getattr(L, name).restype = _I
    _lib = L
    return L


def plane_group_images(nsg: int, ma: int, mb: int, na: int, nb: int, x: float, y: float):
    """Orbit of one atom under plane group nsg (strfac.f90:15-64); CPU-side utility."""
    out = np.zeros(24, dtype=np.float64)
    cnt = ctypes.c_int(0)
    rc = load().trhepd_plane_group_images(nsg, ma, mb, na, nb, x, y, out.ctypes.data,
                                          ctypes.byref(cnt))
    if rc:
        raise TrhepdError(rc, "plane_group_images")
    return out[: 2 * cnt.value].reshape(-1, 2)


class Context:
    """One device context: stream, cached device buffers, options."""

    def __init__(self, device: int = 0):
        L = load()
        h = _P()
        rc = L.trhepd_create(device, ctypes.byref(h))
        if rc:
            raise NativeUnavailable(f"trhepd_create(device={device}) failed with status {rc}")
        self._h = h
        self._L = L

    def _check(self, rc: int):
        if rc:
            raise TrhepdError(rc, self._L.trhepd_last_error(self._h).decode())

    def set_option(self, option: int, value: float):
        self._check(self._L.trhepd_set_option(self._h, option, float(value)))

    def last_stats(self) -> dict:
        out = np.zeros(9)
        self._check(self._L.trhepd_last_stats(self._h, out.ctypes.data, 9))
        return {"renormalisations": int(out[0]), "stage_products": int(out[1]),
                "device_ms": float(out[2]), "stage_columns": int(out[3]),
                "stage_kernel_ms": float(out[4]), "launches": int(out[5]),
                "renorm_launches": int(out[6]), "tensor_kernel_ms": float(out[7]),
                "renorm_ms": float(out[8])}

    def last_curve_errors(self, nangles: int) -> np.ndarray:
        """(nangles, 3) per-curve errors of the last validated split solve: max relative
        error over every spot, max error over the curve maximum, the curve maximum."""
        out = np.zeros(3 * nangles)
        self._check(self._L.trhepd_last_curve_errors(self._h, out.ctypes.data, out.size))
        return out.reshape(nangles, 3)

    def surf_run(self, bulkp, surf, dz2: float, int_method: int = 5, precision: int = FP64,
                 out_path=None):
        """surf.exe for domain 1: returns (f2[nangles, nb], dims)."""
        dims = (ctypes.c_int * 4)()
        # first call sizes the output from the files: nb * naz * ng <= 200*200*nb bound
        cap = 1 << 22
        f2 = np.zeros(cap, dtype=np.float64)
        rc = self._L.trhepd_surf_run(self._h, str(bulkp).encode(), str(surf).encode(),
                                     float(dz2), int(int_method), int(precision),
                                     None if out_path is None else str(out_path).encode(),
                                     f2.ctypes.data, cap, dims)
        self._check(rc)
        nb, nang = dims[0], dims[1]
        return f2[: nb * nang].reshape(nang, nb).copy(), {
            "nb": nb, "nangles": nang, "ns": dims[2], "nv": dims[3]}

    def bulk_run(self, bulk_txt, out_path) -> dict:
        """bulk.exe on the GPU: bulk.txt -> bulkP.b."""
        st = np.zeros(4)
        self._check(self._L.trhepd_bulk_run(self._h, str(bulk_txt).encode(),
                                            str(out_path).encode(), st.ctypes.data))
        return {"device_ms": float(st[0]), "layers": int(st[1]), "double_angle_steps": int(st[2]),
                "items": int(st[3])}

    def rocking_convolution(self, angle_deg, f2, omega: float = 0.5, scan: int | None = None):
        """Gaussian convolution of rocking curves on the GPU (make_convolution.py)."""
        ang = np.ascontiguousarray(angle_deg, dtype=np.float64)
        f = np.ascontiguousarray(f2, dtype=np.float64)
        out = np.zeros_like(f)
        rows, nb = f.shape
        self._check(self._L.trhepd_rocking_convolution(self._h, ang.ctypes.data, f.ctypes.data,
                                                       rows, int(scan or rows), nb,
                                                       float(omega), out.ctypes.data))
        return out

    def close(self):
        if getattr(self, "_h", None):
            self._L.trhepd_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
