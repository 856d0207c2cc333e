"""Continuous-batching request loop for structure-refinement traffic.

Requests are candidate surfaces (a base structure with jittered surface atoms)
with their own beam count N and glancing-angle grid.  The server keeps `slots`
solver contexts, each with its own CUDA stream; a request is admitted when a
slot is free and its device bytes fit the memory budget, so requests arriving
while others run are started at once and their kernels overlap on the device.
Each admitted request gets a device-resident problem (stage table, boundary
data; trhepd_problem_*), is solved, and its intensities are returned.  The
bulk boundary of a (base structure, angle grid) is written once and reused by
every candidate of that base.

Scheduling keeps small requests from queueing behind large ones.  Each slot
serves one range of beam counts and owns one stream of a fixed priority (the
default layout: two slots for N <= 95 at the highest priority, one for
96..191, one for N >= 192 at the lowest); a free slot takes the smallest
pending request of its range.  Streams are created once per slot: a stream
made per request would be mapped round-robin onto the GPU's few hardware work
queues and could land on the queue of a running large solve, behind all of its
queued kernels.  Requests with N <= 64 run the fused FP64 kernel whatever the
server's precision (one launch per solve, exact FP64); larger ones use the
server's precision form.

Latency is completion minus arrival; the report gives p50/p99 and angle-solves/s.
"""
from __future__ import annotations

import dataclasses
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

from . import bulkfile, generator, native, surface

DEFAULT_MIX = {23: 0.30, 47: 0.30, 95: 0.20, 191: 0.15, 521: 0.05}
GRIDS = (31, 61, 121)


@dataclasses.dataclass
class Request:
    rid: int
    n: int
    n_angles: int
    sigma: float
    seed: int
    arrival: float = 0.0          # seconds from stream start
    # filled by the server
    start: float = 0.0
    finish: float = 0.0
    f2: np.ndarray | None = None
    error: str | None = None
    device_ms: float = 0.0

    @property
    def latency(self) -> float:
        return self.finish - self.arrival


def base_structure(n: int, n_angles: int, region: float, dz: float) -> generator.Structure:
    return generator.dense(n, seed=11, n_angles=n_angles, region=region, dz=dz)


def poisson_stream(rate: float, duration: float, seed: int = 0, mix=None,
                   grids=GRIDS) -> list[Request]:
    """Poisson arrivals (mean `rate` per second) for `duration` seconds."""
    mix = mix or DEFAULT_MIX
    rng = np.random.default_rng(seed)
    ns, ws = list(mix), np.array(list(mix.values()), dtype=float)
    ws /= ws.sum()
    out, t, rid = [], 0.0, 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            return out
        out.append(Request(rid=rid, n=int(rng.choice(ns, p=ws)), n_angles=int(rng.choice(grids)),
                           sigma=float(rng.uniform(0.05, 0.2)), seed=int(rng.integers(1 << 30)),
                           arrival=t))
        rid += 1


FUSED_MAX_N = 64
# slot layout: (smallest N, largest N, stream priority 0 lowest .. 1 highest, SM cap
# of the stage-product kernels, 0 = every SM, -1 = one CTA per tile).  A large
# solve's stage kernels hold their SMs for a whole launch (persistent split kernels)
# or a block's lifetime (FP64), so a small request's kernels would queue for SMs
# behind every launch; the large-N slot is capped at 48 of the 148 SMs and the
# other slots always find SMs free.  Their own kernels are not capped: the split
# kernels' CTAs take tiles from a shared counter, so the CTAs that start at once do
# the work.  Three slots serve N <= 95, so a small request rarely waits for a free
# slot of its size class.  (One CTA per tile in the middle slot left the measured
# p99 unchanged; the third small slot lowered it.)
DEFAULT_SLOTS = ((0, 95, 1.0, 0), (0, 95, 1.0, 0), (0, 95, 1.0, 0), (96, 191, 0.5, 0),
                 (192, 1 << 30, 0.0, 48))


class _Pending:
    """Pending requests; a worker serving beam counts lo..hi takes the smallest
    pending request in that range (oldest first among equals)."""

    def __init__(self):
        self.items: list = []
        self.cv = threading.Condition()
        self.unfinished = 0
        self.closing = False

    def put(self, r) -> None:
        with self.cv:
            if r is None:
                self.closing = True
            else:
                self.items.append(r)
                self.unfinished += 1
            self.cv.notify_all()

    def get(self, lo: int = 0, hi: int = 1 << 30):
        with self.cv:
            while True:
                pick = None
                for r in self.items:
                    if lo <= r.n <= hi and (pick is None or r.n < pick.n):
                        pick = r
                if pick is not None:
                    self.items.remove(pick)
                    return pick
                if self.closing:
                    return None
                self.cv.wait(timeout=0.5)

    def task_done(self, r) -> None:
        with self.cv:
            self.unfinished -= 1
            self.cv.notify_all()

    def join(self) -> None:
        with self.cv:
            while self.unfinished:
                self.cv.wait(timeout=0.5)


class Server:
    def __init__(self, device: int = 0, slots=DEFAULT_SLOTS, mem_budget_gb: float = 120.0,
                 precision: int = native.FP64, region: float = 15.0, dz: float = 0.02,
                 renorm_policy: int = 1, schedules: dict | None = None):
        """`slots`: a sequence of (smallest N, largest N, stream priority[, CTA cap])
        per slot, or an int k for k slots that take any request at the default priority.
        `schedules`: an autotune table (N -> chosen schedules); a request uses the
        entry of the nearest tuned N, else the fixed rule of precision_for."""
        self.schedules = schedules
        if isinstance(slots, int):
            slots = tuple((0, 1 << 30, 0.0) for _ in range(slots))
        self.layout = tuple(tuple(s) + (0,) * (4 - len(s)) for s in slots)
        self.slots = len(self.layout)
        self.device, self.precision = device, precision
        self.region, self.dz = region, dz
        self.budget = mem_budget_gb * 1e9
        self.in_use = 0.0
        self.cv = threading.Condition()
        self.q = _Pending()
        self.tmp = Path(tempfile.mkdtemp(prefix="trhepd_serve_"))
        self.bulk_cache: dict = {}
        self.bulk_lock = threading.Lock()
        self.t0 = time.perf_counter()
        self.ctxs = [native.Context(device) for _ in self.layout]
        for c, (_, _, prio, cap) in zip(self.ctxs, self.layout):
            c.set_option(native.OPT_RENORM_POLICY, renorm_policy)
            c.set_option(native.OPT_STREAM_PRIORITY, prio)
            c.set_option(native.OPT_MAX_CTAS, cap)
        self.workers = [threading.Thread(target=self._work, args=(c, lo, hi), daemon=True)
                        for c, (lo, hi, _, _) in zip(self.ctxs, self.layout)]
        self.done: list[Request] = []
        for w in self.workers:
            w.start()

    # ---- inputs
    def _bulk(self, n: int, n_angles: int) -> tuple[generator.Structure, Path]:
        key = (n, n_angles)
        with self.bulk_lock:
            if key not in self.bulk_cache:
                base = base_structure(n, n_angles, self.region, self.dz)
                d = self.tmp / f"base_{n}_{n_angles}"
                base.write(d)
                bulkfile.write_bulkp(base, d / "bulkP.b")
                self.bulk_cache[key] = (base, d / "bulkP.b")
            return self.bulk_cache[key]

    def _inputs(self, r: Request) -> tuple[Path, Path, float]:
        base, bulkp = self._bulk(r.n, r.n_angles)
        cand = generator.jitter(base, r.sigma, r.seed)
        d = self.tmp / f"req_{r.rid}"
        cand.write(d)
        return bulkp, d / "surf.txt", base.surface_dz

    @staticmethod
    def device_bytes(n: int, n_angles: int, nv: int, ncol: int) -> float:
        ld = -(-n // 16) * 16
        state = 3 * n_angles * n * ld * 16
        table = ncol * nv * 32
        split = 6 * n_angles * n * 2 * ld * 4  # digit slices, up to 6 per operand
        return state + table + split + n_angles * n * n * 16

    # ---- scheduling
    def submit(self, r: Request) -> None:
        self.q.put(r)

    def _admit(self, need: float) -> None:
        with self.cv:
            while self.in_use + need > self.budget and self.in_use > 0:
                self.cv.wait(timeout=1.0)
            self.in_use += need

    def _release(self, need: float) -> None:
        with self.cv:
            self.in_use -= need
            self.cv.notify_all()

    def precision_for(self, n: int) -> int:
        """The form a request of n beams runs in: fused FP64 up to 64 beams."""
        return native.FP64 if n <= FUSED_MAX_N else self.precision

    def _configure(self, ctx: native.Context, n: int) -> int:
        """Set the slot context for a request of n beams; returns its precision."""
        if not self.schedules:
            ctx.set_option(native.OPT_FUSED_MAX_N, FUSED_MAX_N)
            return self.precision_for(n)
        from . import autotune
        near = min(self.schedules, key=lambda k: abs(k - n))
        entry = self.schedules[near]
        name = entry["fp64"] if self.precision == native.FP64 else entry["split"]
        return autotune.apply(ctx, autotune.schedule_by_name(name))

    def _work(self, ctx: native.Context, lo: int, hi: int) -> None:
        while True:
            r = self.q.get(lo, hi)
            if r is None:
                return
            need = 0.0
            try:
                bulkp, surf, dz = self._inputs(r)
                sp = surface.SurfaceProblem(ctx, bulkp, surf, dz, 5)
                need = self.device_bytes(sp.args.nb, sp.n_angles, sp.pot.nv,
                                         6 * sp.args.ns + 1)
                self._admit(need)
                r.start = time.perf_counter() - self.t0
                rp = sp.resident()
                rp.solve(self._configure(ctx, r.n))
                r.device_ms = ctx.last_stats()["device_ms"]
                _, r.f2 = rp.fetch()
                rp.close()
                sp.close()
            except Exception as e:  # reported per request
                r.error = str(e)
            finally:
                if need:
                    self._release(need)
                r.finish = time.perf_counter() - self.t0
                with self.cv:
                    self.done.append(r)
                self.q.task_done(r)

    def close(self) -> None:
        self.q.put(None)
        for w in self.workers:
            w.join(timeout=600)
        for c in self.ctxs:
            c.close()


def run_stream(server: Server, stream: list[Request], time_scale: float = 1.0) -> dict:
    """Replay arrivals in real time (scaled), wait for all, and summarise."""
    server.t0 = time.perf_counter()
    for r in stream:
        delay = r.arrival * time_scale - (time.perf_counter() - server.t0)
        if delay > 0:
            time.sleep(delay)
        r.arrival = time.perf_counter() - server.t0
        server.submit(r)
    server.q.join()
    wall = time.perf_counter() - server.t0
    return summarize(stream, wall)


def summarize(stream: list[Request], wall: float) -> dict:
    ok = [r for r in stream if r.error is None and r.finish > 0]
    lat = np.array([r.latency for r in ok]) if ok else np.zeros(1)
    angles = sum(r.n_angles for r in ok)
    by_n = {}
    for n in sorted({r.n for r in ok}):
        ln = np.array([r.latency for r in ok if r.n == n])
        by_n[n] = {"count": int(len(ln)), "p50_s": float(np.percentile(ln, 50)),
                   "p99_s": float(np.percentile(ln, 99))}
    return {"requests": len(stream), "completed": len(ok),
            "errors": len(stream) - len(ok), "wall_s": wall,
            "angle_solves_per_s": angles / wall if wall > 0 else 0.0,
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "by_n": by_n}


def isolated_times(server: Server, cases: list[tuple[int, int]], reps: int = 1) -> dict:
    """Latency of each (N, angle grid) request solved alone on an idle server
    (best of `reps`; the inputs of the base structure are prepared beforehand)."""
    out = {}
    for n, g in cases:
        server._bulk(n, g)
        best = None
        for k in range(reps):
            r = Request(rid=10**9 + len(out) * 10 + k, n=n, n_angles=g, sigma=0.1, seed=k)
            t0 = time.perf_counter()
            r.arrival = t0 - server.t0
            server.submit(r)
            server.q.join()
            if r.error is not None:
                raise RuntimeError(f"isolated request N={n} grid={g}: {r.error}")
            dt = time.perf_counter() - t0
            best = dt if best is None else min(best, dt)
        out[(n, g)] = best
    return out


def slowdowns(stream: list[Request], isolated: dict) -> dict:
    """Latency in the mix over the isolated solve time of the same (N, grid)."""
    ratios = np.array([r.latency / isolated[(r.n, r.n_angles)] for r in stream
                       if r.error is None and r.finish > 0 and (r.n, r.n_angles) in isolated])
    if not len(ratios):
        return {"count": 0}
    return {"count": int(len(ratios)), "p50": float(np.percentile(ratios, 50)),
            "p99": float(np.percentile(ratios, 99)), "max": float(ratios.max())}


def expected_busy_seconds(isolated: dict, mix=None, grids=GRIDS) -> float:
    """Mean isolated solve time of one request drawn from the mix."""
    mix = mix or DEFAULT_MIX
    tot = sum(mix.values())
    return sum(w / tot * np.mean([isolated[(n, g)] for g in grids]) for n, w in mix.items())
