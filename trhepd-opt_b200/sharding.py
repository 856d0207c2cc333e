"""Angle sharding of one srfref problem across ranks (one process per GPU).

Every (azimuth, glancing angle) solve is independent (sim-trhepd-rheed/src/
surflf.f90:79-153 runs them as an OpenMP loop), so a problem splits by the
inner scan index with no exchange during the solve.  Each rank solves a
contiguous block of the inner scan for every outer index; rank 0 gathers the
intensities (nb doubles per angle) over torch.distributed.  `bench.py --gpus N`
uses independent replicas instead (weak scaling); this module is for one large
scan spread over several GPUs.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class Shard:
    start: int   # first inner index (0-based)
    stop: int    # one past the last inner index

    @property
    def count(self) -> int:
        return self.stop - self.start


def shard_inner(nrep2: int, world: int, rank: int) -> Shard:
    """Contiguous, balanced block of the inner scan for `rank`."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    base, extra = divmod(nrep2, world)
    start = rank * base + min(rank, extra)
    return Shard(start, start + base + (1 if rank < extra else 0))


def flat_indices(nrep1: int, nrep2: int, sh: Shard) -> np.ndarray:
    """Flattened angle indices t = irep1 * nrep2 + irep2 covered by a shard."""
    return np.array([r1 * nrep2 + r2 for r1 in range(nrep1) for r2 in range(sh.start, sh.stop)],
                    dtype=np.int64)


def sub_scan(azi: float, daz: float, naz: int, gi: float, dg: float, ng: int, sh: Shard):
    """srfref scan arguments of a shard: the longer scan is the inner loop
    (surflf.f90:43-49); its start and count change, the outer scan is kept."""
    if ng > naz:
        return azi, daz, naz, gi + sh.start * dg, dg, sh.count
    return azi + sh.start * daz, daz, sh.count, gi, dg, ng


def gather_to_root(local: np.ndarray, nrep1: int, nrep2: int, nb: int, world: int, rank: int,
                   group=None) -> np.ndarray | None:
    """Gather every rank's (nrep1 * count, nb) block into the full (nrep1*nrep2, nb)
    array on rank 0 (None elsewhere)."""
    import torch
    import torch.distributed as dist
    sh = shard_inner(nrep2, world, rank)
    maxrows = nrep1 * (nrep2 // world + (1 if nrep2 % world else 0))
    buf = torch.zeros((maxrows, nb), dtype=torch.float64)
    buf[: local.shape[0]] = torch.from_numpy(np.ascontiguousarray(local))
    parts = [torch.zeros_like(buf) for _ in range(world)] if rank == 0 else None
    dist.gather(buf, parts, dst=0, group=group)
    if rank != 0:
        return None
    out = np.zeros((nrep1 * nrep2, nb))
    for r in range(world):
        s = shard_inner(nrep2, world, r)
        idx = flat_indices(nrep1, nrep2, s)
        out[idx] = parts[r][: len(idx)].numpy()
    del sh
    return out
