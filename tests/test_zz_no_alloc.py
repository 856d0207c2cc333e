"""The allocation-free table entry point against the regular one.

trhepd_potential_table_noalloc serves hosts that cannot call cudaMalloc (their
device memory is owned by their own pool or planned once at start-up); it keeps
its device scratch in a fixed array inside the library.  Two calls in a row must
reproduce trhepd_potential_table's tables (same kernel, same inputs), the second
call overwriting the first call's scratch.  This file is collected last.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_tables_match_regular_entry_point(golden):
    from trhepd_opt_b200 import build, native, surface
    build.build()
    L = native.load()
    with native.Context(0) as ctx:
        sp = surface.SurfaceProblem(ctx, golden / "test23" / "bulkP.b",
                                    golden / "test23" / "surf.txt", 0.1, 5)
        v_ref, vi_ref = sp.potential_table(5)
        ncol, nv = v_ref.shape
        for call in range(2):
            v = np.full_like(v_ref, np.nan)
            vi = np.full_like(vi_ref, np.nan)
            nc = ctypes.c_int(0)
            rc = L.trhepd_potential_table_noalloc(ctypes.byref(sp.pot), 5, sp.args.ns,
                                                   sp.args.dz, v.ctypes.data, vi.ctypes.data,
                                                   ctypes.byref(nc))
            assert rc == 0, (call, rc)
            assert nc.value == ncol
            scale = np.abs(v_ref).max()
            assert np.abs(v - v_ref).max() <= 1e-14 * scale, call
            assert np.abs(vi - vi_ref).max() <= 1e-14 * scale, call
        # the other integrators' tables through the same scratch
        for method in (6, 1, 2, 4, 7):
            vm_ref, _ = sp.potential_table(method)
            vm = np.zeros_like(vm_ref)
            nc = ctypes.c_int(0)
            rc = L.trhepd_potential_table_noalloc(ctypes.byref(sp.pot), method, sp.args.ns,
                                                   sp.args.dz, vm.ctypes.data, None,
                                                   ctypes.byref(nc))
            assert rc == 0 and nc.value == vm_ref.shape[0], (method, rc)
            assert np.abs(vm - vm_ref).max() <= 1e-14 * np.abs(vm_ref).max(), method
        # an int_method the reference does not define
        nc = ctypes.c_int(0)
        rc = L.trhepd_potential_table_noalloc(ctypes.byref(sp.pot), 9, sp.args.ns, sp.args.dz,
                                               None, None, ctypes.byref(nc))
        assert rc == 1  # TRHEPD_EINVAL


def test_noalloc_rejects_tables_beyond_its_scratch(golden):
    from trhepd_opt_b200 import native, surface
    L = native.load()
    with native.Context(0) as ctx:
        sp = surface.SurfaceProblem(ctx, golden / "test521" / "bulkP.b",
                                    golden / "test521" / "surf.txt", 0.01, 5)
        # 5947 stage columns x 4755 components x 32 bytes is far beyond 32 MiB
        nc = ctypes.c_int(0)
        rc = L.trhepd_potential_table_noalloc(ctypes.byref(sp.pot), 5, sp.args.ns, sp.args.dz,
                                               None, None, ctypes.byref(nc))
        assert rc == 5  # TRHEPD_ENOMEM
