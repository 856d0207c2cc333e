"""Multi-domain surf.exe on the GPU (NDOM > 1: each domain's srfref at azimuth
azi + rdom, then the weighted sum of the rotated domains, domainsum.f90, on the
device) against the oracle's per-domain solves and its restatement of
domainsum, on a two-domain variant of the reference's N = 23 case
(tests/domain_inputs.py).  The .md file (every domain's rows) and the summed .s
file (E12.4 rows) must read back to the same values."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import spot_errors
from domain_inputs import two_domain_inputs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from trhepd_opt_b200 import build, native
    build.build()
    c = native.Context(0)
    c.set_option(native.OPT_RENORM_POLICY, 0)
    yield c
    c.close()


@pytest.mark.parametrize("precision", [0, 2], ids=["fp64", "int8"])
def test_domain_sum_matches_oracle(ctx, golden, oracle_mod, tmp_path, precision):
    from trhepd_opt_b200 import formats
    bulk, surf = two_domain_inputs(golden, tmp_path)
    oracle_mod.bulk_run(bulk, tmp_path / "bulkP.b")
    out = tmp_path / "surf-bulkP.s"
    f2, dims = ctx.surf_run(tmp_path / "bulkP.b", surf, 0.68, 5, precision, out_path=out)
    S = oracle_mod.Surface(tmp_path / "bulkP.b", surf, 0.68, 5)
    hdr = oracle_mod.domain_header(S)
    curves = oracle_mod.domain_curves(S)
    S.close()
    ang, s2, idomr = oracle_mod.domain_sum(curves, hdr)
    assert dims["nb"] == 23 and dims["nangles"] == 69
    abs_err, rel_err = spot_errors(f2, s2)
    if precision == 0:
        assert abs_err <= 1e-10 and rel_err <= 1e-9, (abs_err, rel_err)
    else:
        assert abs_err <= 1e-8, abs_err
    # the .md file: every domain's rows as srfref writes them
    doms, mh = formats.read_domain_curves(tmp_path / "surf-bulkP.md")
    assert mh["ndom"] == 2 and mh["nbd"] == [23, 23] and mh["rdom_deg"] == [0.0, 60.0]
    assert mh["wdom"] == [0.6, 0.4]
    for (a_f, f_f), (a_o, f_o) in zip(doms, curves):
        np.testing.assert_allclose(a_f, a_o, atol=5e-5)
        assert spot_errors(f_f, f_o)[0] <= (1e-10 if precision == 0 else 1e-8)
    # the summed .s file: E12.4 rows, the reference domain's beams
    a_s, f_s, sh = formats.read_rocking_curves(out)
    assert sh["nb"] == 23 and f_s.shape == s2.shape
    np.testing.assert_allclose(f_s, s2, rtol=5.1e-4, atol=1e-300)  # 4 significant digits
    np.testing.assert_allclose(a_s, ang, atol=5e-5)


def test_bulk_two_domains_matches_oracle(ctx, golden, oracle_mod, tmp_path):
    """bulk.exe with NDOM = 2 on the GPU: header records and both domains' beam
    tables byte-identical to the oracle's file, reflection records to rounding;
    the surface run on the GPU's file equals the run on the oracle's."""
    import struct

    bulk, surf = two_domain_inputs(golden, tmp_path)
    ours, theirs = tmp_path / "gpu.b", tmp_path / "oracle.b"
    st = ctx.bulk_run(bulk, ours)
    assert st["items"] == 2 * 69 * 7
    oracle_mod.bulk_run(bulk, theirs)

    def records(path):
        b = open(path, "rb").read()
        out, p = [], 0
        while p < len(b):
            n = struct.unpack("<i", b[p:p + 4])[0]
            out.append(b[p + 4:p + 4 + n])
            p += 8 + n
        return out
    mine, ref = records(ours), records(theirs)
    assert len(mine) == len(ref)
    worst = 0.0
    for x, y in zip(mine, ref):
        if x == y:
            continue
        xa, ya = np.frombuffer(x, np.complex128), np.frombuffer(y, np.complex128)
        worst = max(worst, float(np.abs(xa - ya).max() / np.abs(ya).max()))
    assert worst <= 1e-9, worst
    fa, _ = ctx.surf_run(ours, surf, 0.68, 5, 0)
    fb, _ = ctx.surf_run(theirs, surf, 0.68, 5, 0)
    assert spot_errors(fa, fb)[0] <= 1e-8
