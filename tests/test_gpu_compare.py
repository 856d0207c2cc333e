"""compare.py's curve metric reduced on the device (trhepd_problem_compare): the
reference's N=23 case solved on the GPU and compared with its converged curves
reproduces the values the reference's runs printed (perf-comp-acc.txt), and
equals the oracle's restatement applied to the fetched curves."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from trhepd_opt_b200 import build, native
    build.build()
    c = native.Context(0)
    c.set_option(native.OPT_RENORM_POLICY, 0)
    yield c
    c.close()


@pytest.mark.parametrize("method", [4, 5, 6, 7])
def test_device_compare_reproduces_reference_rows(ctx, golden, oracle_mod, method):
    from trhepd_opt_b200 import native, surface
    d = golden / "test23"
    acc = np.load(d / "accurate.npz")
    rows = acc[f"comp-{method}-0.68"]
    sp = surface.SurfaceProblem(ctx, d / "bulkP.b", d / "surf.txt", 0.68, method)
    rp = sp.resident()
    rp.solve(native.FP64)
    got = rp.compare(acc["f2"])
    _, f2 = rp.fetch()
    rp.close()
    sp.close()
    # same curves: the device reduction equals the restatement up to summation order
    np.testing.assert_allclose(got, oracle_mod.compare_curves(f2, acc["f2"]), rtol=1e-12)
    # the GPU curves equal the reference's to ~1e-13, the printed errors are ~1e-5
    np.testing.assert_allclose(got, rows[:, 1:], rtol=1e-6, atol=0)


def test_device_compare_rejects_wrong_shape(ctx, golden):
    from trhepd_opt_b200 import native, surface
    d = golden / "test23"
    sp = surface.SurfaceProblem(ctx, d / "bulkP.b", d / "surf.txt", 0.68, 5)
    rp = sp.resident()
    rp.solve(native.FP64)
    with pytest.raises(ValueError):
        rp.compare(np.zeros((3, 3)))
    rp.close()
    sp.close()
