"""Continuous batching: requests solved concurrently on several slots give the
same intensities as the same requests solved alone (the kernels are
deterministic, so the bar is exact equality)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_results_same_alone_and_in_the_mix():
    from trhepd_opt_b200 import build, native, serving
    build.build()
    reqs = [serving.Request(rid=i, n=n, n_angles=g, sigma=0.1, seed=100 + i)
            for i, (n, g) in enumerate([(23, 31), (47, 31), (23, 61), (47, 61), (95, 31),
                                        (23, 31)])]
    srv = serving.Server(slots=3, mem_budget_gb=120.0, region=6.0, dz=0.05)
    try:
        alone = {}
        for r in reqs:
            solo = serving.Request(rid=1000 + r.rid, n=r.n, n_angles=r.n_angles, sigma=r.sigma,
                                   seed=r.seed)
            srv.submit(solo)
            srv.q.join()
            assert solo.error is None, solo.error
            alone[r.rid] = solo.f2
        stats = serving.run_stream(srv, reqs)
    finally:
        srv.close()
    assert stats["completed"] == len(reqs), stats
    for r in reqs:
        assert r.error is None, r.error
        np.testing.assert_array_equal(r.f2, alone[r.rid])
    # requests overlapped: some request started before another finished
    spans = sorted((r.start, r.finish) for r in reqs)
    assert any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))


def test_admission_respects_budget():
    from trhepd_opt_b200 import native, serving
    srv = serving.Server(slots=3, mem_budget_gb=0.001, region=4.0, dz=0.05)
    try:
        reqs = [serving.Request(rid=i, n=23, n_angles=31, sigma=0.1, seed=i) for i in range(4)]
        stats = serving.run_stream(srv, reqs)
    finally:
        srv.close()
    assert stats["completed"] == 4
    # with a budget below one request, requests run one at a time
    spans = sorted((r.start, r.finish) for r in reqs)
    assert all(spans[i + 1][0] >= spans[i][1] - 1e-3 for i in range(len(spans) - 1))
