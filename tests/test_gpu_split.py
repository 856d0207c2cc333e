"""Split-precision forms (BF16 or INT8 digit slices on tcgen05, FP64 elsewhere)
against the plain FP64 form and the reference's output, 5 slices per operand.

Bars, relative on every spot (a spot that is exactly zero in FP64 must be zero):
* INT8 (exact INT32 accumulation of 39-bit digit products): 1e-6, the target of
  the split form;
* BF16 (its slice pairs of weight below 2^-16 accumulate in FP32, which caps it
  near 5e-6 at N = 521): 1e-5.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import spot_errors

pytestmark = pytest.mark.gpu

EVERY_SPOT = {1: 1e-5, 2: 1e-6}   # precision form -> every-spot relative bound


def every_spot_rel(got, ref):
    got, ref = np.asarray(got), np.asarray(ref)
    d = np.abs(got - ref)
    m = np.abs(ref)
    return float(np.where(m > 0, d / np.where(m > 0, m, 1.0), np.where(d > 0, np.inf, 0.0)).max())


@pytest.fixture(scope="module")
def ctx():
    from trhepd_opt_b200 import build, native
    build.build()
    c = native.Context(0)
    yield c
    c.close()


def _resident(ctx, tmp_path, s):
    from trhepd_opt_b200 import bulkfile, surface
    s.write(tmp_path)
    bulkfile.write_bulkp(s, tmp_path / "bulkP.b")
    sp = surface.SurfaceProblem(ctx, tmp_path / "bulkP.b", tmp_path / "surf.txt", s.surface_dz,
                                s.int_method)
    return sp, sp.resident()


# (precision form, BF16 kernel variant)
FORMS = {"persistent": (1, 0), "per_tile": (1, 1), "int8": (2, 0)}


@pytest.mark.parametrize("form", sorted(FORMS))
@pytest.mark.parametrize("case", ["small23", "dense95", "dense200"])
def test_split_matches_fp64(ctx, tmp_path, case, form):
    from trhepd_opt_b200 import generator, native
    if case == "small23":
        s = generator.small23()
    elif case == "dense95":
        s = generator.dense(95, n_angles=8, region=6.0)
    else:  # several row and column tiles, a ragged last tile, 13 angles
        s = generator.dense(200, n_angles=13, region=4.0)
    sp, rp = _resident(ctx, tmp_path, s)
    rp.solve(native.FP64)
    _, ref = rp.fetch()
    precision, variant = FORMS[form]
    ctx.set_option(native.OPT_SPLIT_SLICES, 5)
    ctx.set_option(native.OPT_SPLIT_KERNEL, variant)
    try:
        rp.solve(precision)
        _, got = rp.fetch()
    finally:
        ctx.set_option(native.OPT_SPLIT_KERNEL, 0)
    rel = every_spot_rel(got, ref)
    assert rel <= EVERY_SPOT[precision], rel


@pytest.mark.parametrize("precision", [1, 2], ids=["bf16", "int8"])
def test_split_against_reference_output(ctx, golden, precision):
    """The split forms on the reference's own N=47 case at 0.22 A slices."""
    from trhepd_opt_b200 import native
    d = golden / "test47"
    ref = np.load(d / "perf-5-0.22.npz")
    ctx.set_option(native.OPT_SPLIT_SLICES, 5)
    f2, _ = ctx.surf_run(d / "bulkP.b", d / "surf.txt", 0.22, 5, precision)
    rel = every_spot_rel(f2, ref["f2"])
    assert rel <= EVERY_SPOT[precision], rel


@pytest.mark.parametrize("precision,slices", [(1, (3, 4, 5)), (2, (3, 4, 5, 6))],
                         ids=["bf16", "int8"])
def test_more_slices_is_more_accurate(ctx, tmp_path, precision, slices):
    from trhepd_opt_b200 import generator, native
    sp, rp = _resident(ctx, tmp_path, generator.small23())
    rp.solve(native.FP64)
    _, ref = rp.fetch()
    errs = []
    for S in slices:
        ctx.set_option(native.OPT_SPLIT_SLICES, S)
        rp.solve(precision)
        _, got = rp.fetch()
        errs.append(spot_errors(got, ref)[0])
    ctx.set_option(native.OPT_SPLIT_SLICES, 4)
    assert all(a > b for a, b in zip(errs, errs[1:])), errs


def test_split_slice_limits(ctx, tmp_path):
    """INT8 takes 3 to 6 digit slices, BF16 3 to 5 (its FP32 accumulators gain
    nothing from a sixth): clear errors outside, and the context stays usable."""
    from trhepd_opt_b200 import generator, native
    sp, rp = _resident(ctx, tmp_path, generator.small23())
    with pytest.raises(native.TrhepdError):
        ctx.set_option(native.OPT_SPLIT_SLICES, 7)
    ctx.set_option(native.OPT_SPLIT_SLICES, 6)
    try:
        with pytest.raises(native.TrhepdError):
            rp.solve(native.SPLIT_BF16)
        rp.solve(native.SPLIT_INT8)
    finally:
        ctx.set_option(native.OPT_SPLIT_SLICES, 4)
    rp.solve(native.SPLIT_INT8)


@pytest.mark.parametrize("precision", [1, 2], ids=["bf16", "int8"])
@pytest.mark.parametrize("method", [4, 7])
def test_split_other_integrators(ctx, tmp_path, method, precision):
    """The leapfrog and RK4 paths take the same split stage product."""
    from trhepd_opt_b200 import generator, native
    s = generator.small23()
    s.int_method = method
    sp, rp = _resident(ctx, tmp_path, s)
    rp.solve(native.FP64)
    _, ref = rp.fetch()
    ctx.set_option(native.OPT_SPLIT_SLICES, 5)
    rp.solve(precision)
    _, got = rp.fetch()
    rel = every_spot_rel(got, ref)
    assert rel <= EVERY_SPOT[precision], rel


def test_cta_cap_gives_identical_results(ctx, tmp_path):
    """TRHEPD_OPT_MAX_CTAS caps the stage kernels' grids (a serving slot leaving SMs
    to others) or runs the split kernels one CTA per tile (-1): every tile is
    computed by the same code whichever CTA takes it, so the results are
    bit-identical to the uncapped solve."""
    from trhepd_opt_b200 import generator, native
    sp, rp = _resident(ctx, tmp_path, generator.dense(200, n_angles=13, region=2.0))
    ctx.set_option(native.OPT_SPLIT_SLICES, 5)
    ctx.set_option(native.OPT_FUSED_MAX_N, 0)
    for prec in (native.SPLIT_INT8, native.SPLIT_BF16, native.FP64):
        rp.solve(prec)
        _, ref = rp.fetch()
        for cap in (16, -1):  # at most 16 CTAs; one CTA per tile
            ctx.set_option(native.OPT_MAX_CTAS, cap)
            try:
                rp.solve(prec)
                _, got = rp.fetch()
            finally:
                ctx.set_option(native.OPT_MAX_CTAS, 0)
            assert np.array_equal(got, ref), (prec, cap)
    ctx.set_option(native.OPT_FUSED_MAX_N, 64)
