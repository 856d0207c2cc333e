"""Request-stream generation and latency summaries of the serving loop (CPU)."""
from __future__ import annotations

import numpy as np


def test_poisson_stream_rate_and_mix():
    from trhepd_opt_b200 import serving
    s = serving.poisson_stream(rate=200.0, duration=60.0, seed=1)
    assert abs(len(s) - 12000) < 4 * np.sqrt(12000)
    gaps = np.diff([r.arrival for r in s])
    assert abs(gaps.mean() - 1 / 200) < 0.1 / 200
    frac = {n: np.mean([r.n == n for r in s]) for n in serving.DEFAULT_MIX}
    for n, w in serving.DEFAULT_MIX.items():
        assert abs(frac[n] - w) < 0.02
    assert {r.n_angles for r in s} == set(serving.GRIDS)
    assert all(0.05 <= r.sigma <= 0.2 for r in s)


def test_summary_percentiles():
    from trhepd_opt_b200 import serving
    rs = []
    for i in range(100):
        r = serving.Request(rid=i, n=23, n_angles=31, sigma=0.1, seed=i, arrival=0.0)
        r.finish = (i + 1) / 100.0
        rs.append(r)
    s = serving.summarize(rs, wall=1.0)
    assert s["completed"] == 100 and abs(s["p50_s"] - 0.505) < 1e-9
    assert abs(s["p99_s"] - np.percentile([(i + 1) / 100 for i in range(100)], 99)) < 1e-12
    assert s["angle_solves_per_s"] == 3100.0


def test_pending_ranges_and_order():
    """A worker takes the smallest pending request of its beam-count range (oldest
    first among equals) and never one outside it; closing releases idle workers
    once their range is empty."""
    from trhepd_opt_b200 import serving
    q = serving._Pending()
    reqs = [serving.Request(rid=i, n=n, n_angles=31, sigma=0.1, seed=i)
            for i, n in enumerate([521, 95, 23, 191, 23])]
    for r in reqs:
        q.put(r)
    first = q.get(0, 95)
    assert (first.n, first.rid) == (23, 2)
    assert q.get(0, 95).rid == 4
    assert q.get(0, 95).n == 95
    assert q.get(96, 191).n == 191
    assert q.get(192, 1 << 30).n == 521
    q.put(None)
    assert q.get(0, 95) is None
    for r in reqs:
        q.task_done(r)
    q.join()
