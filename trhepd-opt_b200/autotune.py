"""Per-beam-count schedule choice by measurement.

For each beam count N the tuner builds a short representative problem (the
dense generator's structure with N beams, `angles` glancing angles, a thin
surface region) and times every candidate schedule of the library on it:

* FP64: the fused one-launch kernel (N <= 64) and the stacked DMMA path;
* split: the INT8 digit form with 5 and 6 slices per operand and the BF16 form
  (5 slices) with its persistent and per-tile kernels.

A split candidate qualifies only if every spot intensity stays within `max_err`
relative of the FP64 result on the same problem (a spot that is exactly zero in
FP64 must be zero too).  The result maps N to the
fastest FP64 schedule and the fastest qualifying split schedule; `apply` sets a
context's options for one of them.  Timings are device times of the second solve
(the first sizes buffers), so CUDA-graph replays are what is compared.
"""
from __future__ import annotations

import dataclasses
import json
import tempfile
from pathlib import Path

import numpy as np

from . import bulkfile, generator, native, surface


@dataclasses.dataclass(frozen=True)
class Schedule:
    precision: int          # native.FP64 / SPLIT_INT8 / SPLIT_BF16
    fused: bool = False     # FP64 only: the one-launch kernel (N <= 64)
    kernel: int = 0         # BF16 only: 0 persistent, 1 per tile
    slices: int = 5

    @property
    def name(self) -> str:
        if self.precision == native.FP64:
            return "fp64-fused" if self.fused else "fp64-stacked"
        if self.precision == native.SPLIT_INT8:
            return f"int8x{self.slices}"
        return f"bf16x{self.slices}-{'per-tile' if self.kernel else 'persistent'}"


def candidates(n: int) -> list[Schedule]:
    out = [Schedule(native.FP64, fused=False)]
    if 2 <= n <= 64:
        out.append(Schedule(native.FP64, fused=True))
    out += [Schedule(native.SPLIT_INT8, slices=5), Schedule(native.SPLIT_INT8, slices=6),
            Schedule(native.SPLIT_BF16, kernel=0), Schedule(native.SPLIT_BF16, kernel=1)]
    return out


def every_spot_error(f2, ref) -> float:
    """Largest relative error over every spot (0 / 0 counts 0, x / 0 infinity)."""
    d = np.abs(f2 - ref)
    m = np.abs(ref)
    rel = np.where(m > 0, d / np.where(m > 0, m, 1.0), np.where(d > 0, np.inf, 0.0))
    return float(rel.max())


def apply(ctx: native.Context, sch: Schedule) -> int:
    """Set ctx's options for `sch`; returns the precision form to solve with."""
    ctx.set_option(native.OPT_FUSED_MAX_N, 64 if sch.fused else 0)
    ctx.set_option(native.OPT_SPLIT_SLICES, sch.slices)
    ctx.set_option(native.OPT_SPLIT_KERNEL, sch.kernel)
    return sch.precision


def _problem(ctx, n: int, angles: int, region: float, dz: float, workdir: Path):
    s = generator.dense(n, seed=30 + n, n_angles=angles, region=region, dz=dz)
    d = workdir / f"n{n}"
    s.write(d)
    bulkfile.write_bulkp(s, d / "bulkP.b")
    sp = surface.SurfaceProblem(ctx, d / "bulkP.b", d / "surf.txt", s.surface_dz, s.int_method)
    return sp, sp.resident()


def tune(ctx: native.Context, beam_counts=(23, 47, 95, 191, 521), angles: int = 16,
         region: float = 2.0, dz: float = 0.02, max_err: float = 1e-6) -> dict:
    """Time every candidate for each N; returns {N: {"fp64": name, "split": name,
    "times_ms": {name: ms}, "errors": {name: err}}}."""
    workdir = Path(tempfile.mkdtemp(prefix="trhepd_tune_"))
    out = {}
    try:
        for n in beam_counts:
            sp, rp = _problem(ctx, n, angles, region, dz, workdir)
            times, errs, ref = {}, {}, None
            for sch in candidates(n):
                prec = apply(ctx, sch)
                rp.solve(prec)            # sizes buffers
                rp.solve(prec)            # captured / replayed
                times[sch.name] = ctx.last_stats()["device_ms"]
                _, f2 = rp.fetch()
                if sch.precision == native.FP64 and ref is None:
                    ref = f2
                if ref is not None:
                    errs[sch.name] = every_spot_error(f2, ref)
            rp.close()
            sp.close()
            cands = candidates(n)
            fp64 = min((c for c in cands if c.precision == native.FP64),
                       key=lambda c: times[c.name])
            split_ok = [c for c in cands if c.precision != native.FP64
                        and errs.get(c.name, np.inf) <= max_err]
            split = min(split_ok, key=lambda c: times[c.name]) if split_ok else fp64
            # a split form is only worth it where it is faster than the best FP64 one
            if times[split.name] >= times[fp64.name]:
                split = fp64
            out[n] = {"fp64": fp64.name, "split": split.name, "times_ms": times,
                      "errors": errs, "problem": {"angles": angles, "region_A": region,
                                                  "dz_A": dz}}
    finally:
        apply(ctx, Schedule(native.FP64, fused=True))
        ctx.set_option(native.OPT_SPLIT_KERNEL, 0)
    return out


def schedule_by_name(name: str) -> Schedule:
    for n in (23, 521):
        for c in candidates(n):
            if c.name == name:
                return c
    raise KeyError(name)


def save(table: dict, path) -> None:
    Path(path).write_text(json.dumps({str(k): v for k, v in table.items()}, indent=1))


def load(path) -> dict:
    return {int(k): v for k, v in json.loads(Path(path).read_text()).items()}
