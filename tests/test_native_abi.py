"""The C-ABI library loads and exports every symbol include/trhepd_b200.h
declares; the CPU-side plane-group routine matches the oracle's restatement
for all 17 groups (general and special positions)."""
from __future__ import annotations

import ctypes
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_symbols():
    text = (ROOT / "include" / "trhepd_b200.h").read_text()
    return sorted(set(re.findall(r"\b(trhepd_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_header_symbols():
    from trhepd_opt_b200 import build, native
    build.build()
    lib = ctypes.CDLL(str(native.LIB))
    syms = declared_symbols()
    assert len(syms) >= 10
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert set(native.EXPORTS) == set(syms)


def _oracle_images(oracle_mod, nsg, ma, mb, na, nb, x, y):
    L = oracle_mod.lib()
    f = L.oracle_plane_group_images
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int] * 5 + [ctypes.c_double] * 2 + [ctypes.c_void_p]
    out = np.zeros(24)
    n = f(nsg, ma, mb, na, nb, x, y, out.ctypes.data)
    return out[: 2 * n].reshape(-1, 2)


SPECIAL = [(0.0, 0.0), (0.5, 0.5), (0.5, 0.0), (0.0, 0.5), (0.25, 0.25), (0.25, 0.75),
           (1 / 3, 2 / 3), (2 / 3, 1 / 3), (0.3, 0.3), (0.3, 0.0), (0.0, 0.3), (0.2, 0.4),
           (0.4, 0.2), (0.3, 0.8), (0.3, 0.25), (0.1, 0.6), (0.6, 0.9)]


@pytest.mark.parametrize("nsg", list(range(1, 18)))
def test_plane_group_images_match_oracle(oracle_mod, nsg):
    from trhepd_opt_b200 import native
    rng = np.random.default_rng(nsg)
    pts = SPECIAL + [tuple(rng.uniform(-1, 2, 2)) for _ in range(20)]
    for cell in [(1, 0, 0, 1), (2, 0, 0, 2), (7, 0, 0, 7), (2, 1, -1, 1)]:
        for x, y in pts:
            a = native.plane_group_images(nsg, *cell, x, y)
            b = _oracle_images(oracle_mod, nsg, *cell, x, y)
            assert a.shape == b.shape, (nsg, cell, x, y)
            np.testing.assert_allclose(a, b, rtol=0, atol=1e-12)
