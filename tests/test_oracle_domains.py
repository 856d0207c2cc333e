"""The oracle's restatement of the multi-domain sum (domainsum.f90) on a
two-domain variant of the reference's N = 23 case (tests/domain_inputs.py): the
second domain's beams are the first's rotated by 60 deg, so each maps onto the
beam of the same index and the sum is w1 f2_1 + w2 f2_2 beam by beam."""
from __future__ import annotations

import numpy as np

from domain_inputs import two_domain_inputs


def test_domain_sum_restatement(golden, oracle_mod, tmp_path):
    bulk, surf = two_domain_inputs(golden, tmp_path)
    oracle_mod.bulk_run(bulk, tmp_path / "bulkP.b")
    S = oracle_mod.Surface(tmp_path / "bulkP.b", surf, 0.68, 5)
    hdr = oracle_mod.domain_header(S)
    assert hdr["nbd"] == [23, 23] and np.allclose(hdr["wdom"], [0.6, 0.4])
    curves = oracle_mod.domain_curves(S)
    S.close()
    ang, s2, idomr = oracle_mod.domain_sum(curves, hdr)
    f0, f1 = curves[0][1], curves[1][1]
    assert idomr == 0 and s2.shape == f0.shape
    assert np.array_equal(s2, f0 * 0.6 + f1 * 0.4)
    # the domains see different azimuths: their curves differ
    assert np.abs(f0 - f1).max() > 0.1 * np.abs(f0).max()
    # a weight the .md header cannot carry is read back rounded to 3 digits
    hdr2 = dict(hdr, wdom=np.array([0.6, 1.0 / 3.0]))
    _, s3, _ = oracle_mod.domain_sum(curves, hdr2)
    assert np.array_equal(s3, f0 * 0.6 + f1 * 0.333)
