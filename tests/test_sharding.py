"""Angle sharding over two ranks (gloo, CPU): each rank solves its block of the
inner scan and rank 0 gathers; the result equals the unsharded solve.  The
per-rank solver here is the CPU oracle (the checker); on GPUs it is the C ABI."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import GOLDEN


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, outq):
    import sys
    sys.path.insert(0, str(GOLDEN.parents[1]))
    sys.path.insert(0, str(GOLDEN.parents[0]))
    import conftest  # noqa: F401  (loads the package)
    import torch.distributed as dist
    from oracle import oracle as O
    from trhepd_opt_b200 import sharding
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        O.set_threads(2)
        d = GOLDEN / "test23"
        S = O.Surface(d / "bulkP.b", d / "surf.txt", 0.68, 5)
        sh = sharding.shard_inner(S.nrep2, world, rank)
        blocks = [S.solve(r1 * S.nrep2 + sh.start, sh.count)[0] for r1 in range(S.nrep1)]
        local = np.concatenate(blocks, axis=0)
        full = sharding.gather_to_root(local, S.nrep1, S.nrep2, S.nb, world, rank)
        if rank == 0:
            outq.put(full)
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_rank_shards_equal_unsharded():
    from oracle import oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    full = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    d = GOLDEN / "test23"
    ref, _, _ = O.Surface(d / "bulkP.b", d / "surf.txt", 0.68, 5).solve()
    np.testing.assert_array_equal(full, ref)


@pytest.mark.parametrize("nrep2,world", [(69, 2), (61, 4), (3, 4), (121, 8)])
def test_shards_cover_scan(nrep2, world):
    from trhepd_opt_b200 import sharding
    seen = []
    for r in range(world):
        s = sharding.shard_inner(nrep2, world, r)
        seen.extend(range(s.start, s.stop))
    assert seen == list(range(nrep2))


def test_sub_scan_moves_the_inner_scan():
    from trhepd_opt_b200 import sharding
    sh = sharding.Shard(10, 20)
    assert sharding.sub_scan(0.0, 0.0, 1, 0.01, 0.002, 61, sh) == (0.0, 0.0, 1, 0.01 + 10 * 0.002,
                                                                  0.002, 10)
    assert sharding.sub_scan(0.1, 0.05, 40, 0.02, 0.0, 1, sh) == (0.1 + 10 * 0.05, 0.05, 10, 0.02,
                                                                 0.0, 1)
