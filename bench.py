#!/usr/bin/env python
"""Angle-solves/s of the multislice surface solve on B200.

Workload (default ``dense521``): synthetic 2x2 Si/Ge surface over a 4-atom
bulk, N = 521 beams, 61 glancing angles (0.5..6.5 deg), 2004 slices of
0.01 A, symplectic RKN-4 (int_method 5).  One step = one solve of all 61 angles.

* ``value``: the split-precision form (default: 5 signed 8-bit digit slices per
  operand, 39 bits, on tcgen05 kind::i8 with exact INT32 accumulation; every
  spot within 1e-6 relative of FP64 at N = 521; ``--precision``
  bf16 / fp64 select the other forms), inputs resident in HBM
  (trhepd_problem_solve), device time from CUDA events on the library stream,
  max over ranks.
* ``e2e``: the same metric through the C ABI with host buffers
  (trhepd_srfref: uploads, stage-table build, solve, intensities back).
* ``fp64``: the plain FP64 form of the same workload, its speed and the split
  form's error against it; ``bf16_split``: the BF16-slice form beside it.
* ``roofline``: the tensor-core stage kernel, live event timing of every launch.
* ``cpu_baseline``: the CPU oracle (C++ restatement of the reference path,
  OpenMP over angles, OpenBLAS) on a bounded sample of the workload.

Multi-GPU (torchrun): every rank solves its own workload (independent angle
batches, no collective on the data path): weak scaling.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

# more hardware work queues than the default 8, so that the serving slots' streams
# (and torch's) do not share one and serialise behind each other's kernels; read
# when CUDA initialises, so it is set before any CUDA call of this process
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def load_package():
    name = "trhepd_opt_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg = ROOT / "trhepd-opt_b200"
    spec = importlib.util.spec_from_file_location(name, pkg / "__init__.py",
                                                  submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


load_package()
from trhepd_opt_b200 import build as tbuild  # noqa: E402
from trhepd_opt_b200 import bulkfile, generator, native, surface  # noqa: E402

METRIC = "angle-solves/s at N=521, split-precision vs FP64 on 1 B200; p50/p99 latency"
# DRAM bytes (read + write) per launch of the stage kernels from one ncu capture of
# the 16-angle profiling case (dense521s, same N and generator), keyed by (workload,
# form, digit slices); the bench scales them by angles / 16.  Summaries and commands:
# profiles/k_split_gemm_i8_dense521s.md, profiles/k_stage_gemm_f64_dense521s.md.
NCU_TRAFFIC: dict = {
    ("dense521", "int8", 5): (202.690816 + 95.043584) * 1e6,  # k_split_gemm_i8<5>
    ("dense521", "fp64", 0): (145.711360 + 85.679872) * 1e6,  # k_stage_gemm_f64
}
WORKLOADS = {
    "dense521": ("dense521: N=521 beams, 61 glancing angles 0.5-6.5 deg, 20 A region in 0.01 A "
                 "slices (sp4 RKN), synthetic 2x2 Si/Ge surface over 4-atom bulk, seed 3",
                 lambda seed: generator.dense(521, seed=3 + seed)),
    "dense521s": ("dense521s (profiling case): N=521 beams, 16 angles, 4 A region in 0.01 A "
                  "slices (sp4), same generator as dense521",
                  lambda seed: generator.dense(521, n_angles=16, region=4.0, seed=3 + seed)),
    "small23": ("small23: N=23 beams, 61 angles, 15 A region in 0.02 A slices (sp4), seed 1",
                lambda seed: generator.small23(1 + seed)),
    "batch47": ("batch47: N=47 beams, 121 angles x 2 azimuths, 15 A in 0.02 A slices (sp4)",
                lambda seed: generator.batch47(2 + seed)),
}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """nvidia-smi sampler for the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "samples": len(sm), "reasons": sorted(reasons)}


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            pass
    return {}


def library_gemm_peak(device: int, kind: str, seconds: float = 3.0) -> dict | None:
    """Library GEMM 8192^3 throughput in T(FL)OP/s on this GPU: cuBLAS DGEMM (kind
    "f64", the FP64 tensor-core reference) or cuBLASLt INT8 -> INT32 (kind "i8",
    torch._int_mm).  "burst" is the best of 5 single launches, "sustained" the mean
    over a back-to-back loop of `seconds`, the figure for kernels timed inside a
    long solve."""
    try:
        import torch
        torch.cuda.set_device(device)
        n = 8192
        if kind == "f64":
            a = torch.randn(n, n, dtype=torch.float64, device="cuda")
            b = torch.randn(n, n, dtype=torch.float64, device="cuda")
            op = lambda: torch.matmul(a, b)  # noqa: E731
        else:
            a = torch.randint(-128, 128, (n, n), dtype=torch.int8, device="cuda")
            b = torch.randint(-128, 128, (n, n), dtype=torch.int8,
                              device="cuda").t().contiguous().t()
            op = lambda: torch._int_mm(a, b)  # noqa: E731
        for _ in range(3):
            op()
        torch.cuda.synchronize()
        best = 1e30
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            op()
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        reps = max(3, int(seconds * 1e3 / best))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            op()
        e1.record()
        torch.cuda.synchronize()
        mean = e0.elapsed_time(e1) / reps
        del a, b
        torch.cuda.empty_cache()
        w = 2.0 * n ** 3
        return {"burst": w / (best * 1e-3) / 1e12, "sustained": w / (mean * 1e-3) / 1e12}
    except Exception:
        return None


def prepare_inputs(workload: str, seed: int, workdir: Path):
    desc, make = WORKLOADS[workload]
    s = make(seed)
    s.write(workdir)
    # bulk boundary records: non-reflecting bulk (f = 0); the surface-solve work is
    # independent of the record values
    bulkfile.write_bulkp(s, workdir / "bulkP.b")
    return s, desc


def cpu_sample_plan(workdir: Path, s, nangles: int, seconds: float) -> dict:
    """Size a bounded sample of the workload for the oracle on the host cores: all
    threads, one angle per thread, the first L slices with L chosen so that one
    sample takes about `seconds`."""
    from oracle import oracle as O
    O.build()
    cores = O.set_threads(os.cpu_count())
    nang = min(nangles, cores)
    O.set_max_slices(2)
    S = O.Surface(workdir / "bulkP.b", workdir / "surf.txt", s.surface_dz, s.int_method)
    t0 = time.perf_counter()
    S.solve(0, nang)
    t_cal = time.perf_counter() - t0
    S.close()
    O.set_max_slices(0)
    L = max(2, min(2000, int(2 * seconds / max(t_cal, 1e-3))))
    return {"angles": nang, "slices": L, "cores": cores}


def cpu_sample(workdir: Path, s, plan: dict) -> tuple[float, int]:
    """One timed sample: (seconds, slices actually integrated)."""
    from oracle import oracle as O
    O.set_max_slices(plan["slices"])
    S = O.Surface(workdir / "bulkP.b", workdir / "surf.txt", s.surface_dz, s.int_method)
    L = S.ns
    t0 = time.perf_counter()
    S.solve(0, plan["angles"])
    t = time.perf_counter() - t0
    S.close()
    O.set_max_slices(0)
    return t, L


def cpu_model() -> str:
    """The host CPU's model name (Linux /proc/cpuinfo), else the platform's."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def cpu_baseline(workdir: Path, s, nangles: int, reps: int = 5, seconds: float = 6.0) -> dict:
    """The median of `reps` timed samples of about `seconds` each."""
    plan = cpu_sample_plan(workdir, s, nangles, seconds)
    runs = [cpu_sample(workdir, s, plan) for _ in range(reps)]
    times = sorted(t for t, _ in runs)
    return {"seconds": times[len(times) // 2], "samples_s": times, "angles": plan["angles"],
            "slices": runs[0][1], "cores": plan["cores"]}


def serve_leg(device: int, seconds: float, load: float, precision: int, seed: int = 0) -> dict:
    """Poisson stream of mixed-N refinement requests through the serving loop at
    `load` times the throughput the isolated solve times allow; reports p50/p99
    latency, angle-solves/s and each request's latency over its isolated time."""
    from trhepd_opt_b200 import autotune, serving
    tctx = native.Context(device)
    try:
        table = autotune.tune(tctx, beam_counts=tuple(serving.DEFAULT_MIX))
    finally:
        tctx.close()
    srv = serving.Server(device=device, slots=serving.DEFAULT_SLOTS, mem_budget_gb=120.0,
                         precision=precision, schedules=table)
    try:
        cases = [(n, g) for n in serving.DEFAULT_MIX for g in serving.GRIDS]
        iso = serving.isolated_times(srv, cases)
        busy = serving.expected_busy_seconds(iso)
        rate = load / busy
        stream = serving.poisson_stream(rate, seconds, seed=seed)
        out = serving.run_stream(srv, stream)
        out["latency_over_isolated"] = serving.slowdowns(stream, iso)
    finally:
        srv.close()
    out["by_n"] = {str(k): v for k, v in out["by_n"].items()}
    out["schedules"] = {str(n): {"fp64": e["fp64"], "split": e["split"],
                                 "times_ms": e["times_ms"]} for n, e in table.items()}
    out.update({"arrival_rate_req_s": rate, "duration_s": seconds, "target_load": load,
                "mean_isolated_request_s": busy,
                "isolated_s": {f"{n}x{g}": t for (n, g), t in iso.items()},
                "mix": {str(k): v for k, v in serving.DEFAULT_MIX.items()},
                "grids": list(serving.GRIDS),
                "slots": [{"n_min": lo, "n_max": hi, "stream_priority": p, "max_ctas": cap}
                          for lo, hi, p, cap in serving.DEFAULT_SLOTS],
                "hbm_budget_gb": 120.0,
                "structures": "dense(N) base per (N, grid), 15 A region in 0.02 A slices, "
                              "surface atoms jittered by sigma in [0.05, 0.2] A per request"})
    return out


def uneven_leg(ctx, precision: int, per_n: int = 64, seed: int = 0) -> dict:
    """Candidate-structure batch of uneven beam counts: per_n jittered candidates
    (sigma 0.1 A) of a base structure for each N in {23, 47, 95, 191}, 61 angles,
    15 A in 0.02 A slices, all solved by one trhepd_batch_solve (the N <= 64 ones
    in shared fused launches); two batch solves warm up, the next one is timed
    (device time from the library's events).  per_n = 64 is the 256-structure
    candidate batch."""
    tmp = Path(tempfile.mkdtemp(prefix="trhepd_uneven_"))
    probs, nang = [], 0
    for n in (23, 47, 95, 191):
        base = generator.dense(n, seed=20 + n + seed, n_angles=61, region=15.0, dz=0.02)
        for k in range(per_n):
            s = generator.jitter(base, 0.1, 1000 * n + k)
            d = tmp / f"n{n}_{k}"
            s.write(d)
            bulkfile.write_bulkp(s, d / "bulkP.b")
            sp = surface.SurfaceProblem(ctx, d / "bulkP.b", d / "surf.txt", s.surface_dz,
                                        s.int_method)
            probs.append((sp, sp.resident()))
            nang += probs[-1][1].nangles
    rps = [rp for _, rp in probs]
    for _ in range(2):  # buffers sized, graphs of the larger problems captured
        surface.solve_batch(ctx, rps, precision)
    ms = []
    for _ in range(1):
        surface.solve_batch(ctx, rps, precision)
        ms.append(ctx.last_stats()["device_ms"])
    st = ctx.last_stats()
    for sp, rp in probs:
        rp.close()
        sp.close()
    t = sum(ms) / len(ms) / 1e3
    return {"structures": len(probs), "beam_counts": [23, 47, 95, 191], "per_n": per_n,
            "angles_per_structure": 61, "slices": "15 A in 0.02 A", "angle_solves": nang,
            "seconds_per_batch": t, "angle_solves_per_s": nang / t,
            "launches_per_batch": st["launches"],
            "note": "N <= 64 in fused FP64 launches, N = 95, 191 in the requested form"}


def bulk_leg(ctx, cpu: bool) -> dict:
    """The bulk boundary solve (bulk.exe: bulk.txt -> bulkP.b) timed on its own, as
    the reference runs it in a separate program: the reference's N = 23 structure
    (69 angles x 7 beam groups) and N = 521 structure (1 angle x 49 groups), GPU
    device time of the second run, beside the oracle on the host cores."""
    out = {}
    for case in ("test23", "test521"):
        d = ROOT / "tests" / "golden" / case
        tmp = Path(tempfile.mkdtemp(prefix="trhepd_bulk_"))
        ctx.bulk_run(d / "bulk.txt", tmp / "bulkP.b")
        st = ctx.bulk_run(d / "bulk.txt", tmp / "bulkP.b")
        e = {"device_ms": st["device_ms"], "items": st["items"], "layers": st["layers"],
             "item_solves_per_s": st["items"] / (st["device_ms"] / 1e3)}
        if cpu:
            from oracle import oracle as O
            O.build()
            t0 = time.perf_counter()
            O.bulk_run(d / "bulk.txt", tmp / "oracle.b")
            e["oracle_host_s"] = time.perf_counter() - t0
        out[case] = e
    out["note"] = ("(angle, beam group) items; GPU: slice propagators from matrix cos/sin "
                   "series, layer recursion with the reference's convergence exit")
    return out


def rk4_leg(ctx) -> dict:
    """int_method 7 (RK4, Gauss-Jordan renormalisation on the Gershgorin test) and
    int_method 8 (RK4, CholeskyQR when the power estimate exceeds 1e2) on the
    reference's test47 structure (N = 47, 0.22 A slices), plain FP64 through
    trhepd_surf_run: device time of the second solve of each, and how far the two
    results are apart (the re-orthogonalisation changes rounding only)."""
    out = {}
    try:
        d = ROOT / "tests" / "golden" / "test47"
        ctx.set_option(native.OPT_RENORM_POLICY, 0)
        f2s = {}
        for m in (7, 8):
            ctx.surf_run(d / "bulkP.b", d / "surf.txt", 0.22, m, native.FP64)
            f2, dims = ctx.surf_run(d / "bulkP.b", d / "surf.txt", 0.22, m, native.FP64)
            ms = ctx.last_stats()["device_ms"]
            f2s[m] = f2
            out[f"int_method_{m}"] = {"device_ms": ms, "angles": dims["nangles"],
                                      "angle_solves_per_s": dims["nangles"] / (ms / 1e3)}
        rowmax = np.maximum(np.abs(f2s[7]).max(axis=1, keepdims=True), 1e-300)
        out["max_diff_vs_rowmax"] = float((np.abs(f2s[8] - f2s[7]) / rowmax).max())
    except Exception as e:  # a failed leg is reported, the bench line still prints
        out["error"] = f"{type(e).__name__}: {e}"
    finally:
        ctx.set_option(native.OPT_RENORM_POLICY, 1)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="dense521", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="auto", choices=["auto", "int8", "bf16", "fp64"],
                    help="auto: the INT8 split form")
    ap.add_argument("--slices", type=int, default=5,
                    help="digit slices per operand of the split forms (INT8 3..6, BF16 3..5)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-bf16", action="store_true", help="skip the BF16 split comparison")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-uneven", action="store_true", help="skip the uneven candidate batch")
    ap.add_argument("--no-bulk", action="store_true", help="skip the bulk boundary solve leg")
    ap.add_argument("--no-rk4", action="store_true", help="skip the int_method 7/8 leg")
    ap.add_argument("--uneven-per-n", type=int, default=64,
                    help="candidates per beam count in the uneven batch (64: 256 structures)")
    ap.add_argument("--serve-seconds", type=float, default=60.0)
    ap.add_argument("--serve-load", type=float, default=0.5,
                    help="arrival rate as a fraction of the isolated-solve throughput")
    ap.add_argument("--no-serve-fp64", action="store_true",
                    help="skip the serving stream in the plain FP64 form")
    args = ap.parse_args()
    ws, rank, local = dist_env()
    pg = None
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist

    workdir = Path(tempfile.mkdtemp(prefix=f"trhepd_bench_r{rank}_"))
    s, desc = prepare_inputs(args.workload, rank, workdir)

    if args.impl == "reference":
        if rank == 0:
            S_ns = surface_slices(workdir, s)
            plan = cpu_sample_plan(workdir, s, 61, seconds=8.0)
            for _ in range(max(args.warmup, 0)):
                cpu_sample(workdir, s, plan)
            tot, L = 0.0, plan["slices"]
            for _ in range(args.steps):
                t, L = cpu_sample(workdir, s, plan)
                tot += t
            full = tot * S_ns / L  # seconds for the sampled angles over every slice
            value = plan["angles"] * args.steps / full
            line = {"impl": "reference", "metric": METRIC, "value": value,
                    "unit": "angle-solves/s", "n_gpus": args.gpus, "steps": args.steps,
                    "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
                    "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                    "dtype": "f64", "data": "synthetic",
                    "config": {"workload": desc},
                    "cpu_baseline": {"value": value, "unit": "angle-solves/s",
                                     "cores": plan["cores"], "kind": "port",
                                     "cpu_model": cpu_model(), "nproc": os.cpu_count(),
                                     "sample": f"per step {plan['angles']} angles x first {L} "
                                               f"of {S_ns} slices on {plan['cores']} threads, "
                                               "scaled by slice count"},
                    "e2e": {"value": value, "unit": "angle-solves/s",
                            "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
            print(json.dumps(line), flush=True)
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return

    tbuild.build()
    ctx = native.Context(local)
    sp = surface.SurfaceProblem(ctx, workdir / "bulkP.b", workdir / "surf.txt", s.surface_dz,
                                s.int_method)
    rp = sp.resident()
    nang, n = rp.nangles, rp.nb
    ctx.set_option(native.OPT_RENORM_POLICY, 1)
    prec = {"auto": native.SPLIT_INT8, "int8": native.SPLIT_INT8, "bf16": native.SPLIT_BF16,
            "fp64": native.FP64}[args.precision]
    split = prec != native.FP64
    slices = args.slices
    ctx.set_option(native.OPT_SPLIT_SLICES, slices)

    def solve_ms(p):
        rp.solve(p)
        return ctx.last_stats()

    for _ in range(max(args.warmup, 0)):
        solve_ms(prec)
    clocks = Clocks(local)
    if pg:
        pg.barrier()
    clocks.start()
    t_wall = time.perf_counter()
    total_ms, launches = 0.0, 0
    for _ in range(args.steps):
        st = solve_ms(prec)
        total_ms += st["device_ms"]
        launches += st["launches"]
    t_wall = time.perf_counter() - t_wall
    clk = clocks.stop()
    max_ms = total_ms
    if pg:
        import torch
        t = torch.tensor([total_ms], dtype=torch.float64, device=f"cuda:{local}")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        max_ms = float(t.item())
    value = nang * args.steps * ws / (max_ms / 1e3)
    ms_per_step = max_ms / args.steps
    _, f2_main = rp.fetch()

    # ---- roofline of the tensor-core stage kernel (one profiled solve): CUDA events
    # around every launch of that kernel on the library stream
    ctx.set_option(native.OPT_PROFILE, 1)
    stp = solve_ms(prec)
    ctx.set_option(native.OPT_PROFILE, 0)
    nprod = max(stp["stage_products"], 1)
    tensor_ms = stp["tensor_kernel_ms"] / nprod
    stage_ms = stp["stage_kernel_ms"] / nprod
    fp64_equiv = 8.0 * nang * n ** 3  # complex N x N x N product per angle
    pairs = slices * (slices + 1) // 2 if split else 1
    issued = pairs * fp64_equiv       # slice-pair GEMM work of one launch
    achieved = issued / (tensor_ms * 1e-3) / 1e12
    peaks = measured_peaks()
    f64_peak = library_gemm_peak(local, "f64") if rank == 0 else None
    if prec == native.SPLIT_INT8:
        pk = library_gemm_peak(local, "i8") if rank == 0 else None
        peak = pk["sustained"] if pk else None
        peak_src = ("cuBLASLt INT8 GEMM 8192^3 (torch._int_mm) measured in this run, "
                    "sustained over a 3 s loop")
        kernel, unit = "k_split_gemm_i8 (tcgen05 kind::i8, INT32 accumulators)", "TOP/s"
    elif prec == native.SPLIT_BF16:
        pk = None
        peak = peaks.get("bf16_tflops_sustained") or 1400.0
        peak_src = ("MEASURED_PEAKS.json bf16_tflops_sustained (of measured)" if peaks else
                    "fallback 1.4 PFLOP/s sustained")
        kernel, unit = "k_split_gemm_p (tcgen05 kind::f16, FP32 accumulators)", "TFLOP/s"
    else:
        pk = None
        peak = f64_peak["sustained"] if f64_peak else None
        peak_src = "cuBLAS DGEMM 8192^3 measured in this run, sustained over a 3 s loop"
        kernel, unit = "k_stage_gemm_f64 (FP64 DMMA)", "TFLOP/s"
    fp64_equiv_tflops = fp64_equiv / (tensor_ms * 1e-3) / 1e12
    form = args.precision if args.precision != "auto" else "int8"
    # the two rooflines of the stage kernel: issued tensor work and algorithmic HBM
    # bytes (state Q, P read; P, Q' written; digit slices A and B read once)
    ld = -(-n // 16) * 16
    kc = ld
    hbm_bytes = 4 * 16.0 * nang * n * n
    if split:
        hbm_bytes += (slices if prec == native.SPLIT_INT8 else 2 * slices) * nang * n * 2 * kc
    hbm_peak = peaks.get("hbm_gbs") or 6650.0
    hbm_ms = hbm_bytes / (hbm_peak * 1e9) * 1e3
    # INT8: the tcgen05 kind::i8 issue rate measured by a back-to-back MMA probe on
    # this part, 8192 MAC per clock per SM, at the median SM clock of the timed region
    mma_issue = None
    if prec == native.SPLIT_INT8 and clk.get("sm_mhz"):
        try:
            import torch
            sms = torch.cuda.get_device_properties(local).multi_processor_count
        except Exception:
            sms = 148
        mma_issue = 2 * 8192 * sms * clk["sm_mhz"] * 1e6 / 1e12   # TOP/s
    traffic = NCU_TRAFFIC.get((args.workload, form, slices))
    tensor_floor_ms = issued / (peak * 1e12) * 1e3 if peak else 0.0
    roof = {"bound": "tensor" if tensor_floor_ms >= hbm_ms else "hbm",
            "achieved": achieved, "peak": peak, "unit": unit,
            "frac": (achieved / peak) if peak else None,
            "traffic": (traffic * nang / 16.0) if traffic else None,
            "kernel": kernel, "peak_source": peak_src, "library_peak": pk,
            "avg_launch_ms": tensor_ms, "stage_product_ms": stage_ms, "ops_per_launch": issued,
            "slice_pairs": pairs, "fp64_equivalent_tflops": fp64_equiv_tflops,
            "fp64_library_peak_tflops": f64_peak,
            "frac_of_fp64_peak": (fp64_equiv_tflops / f64_peak["sustained"]) if f64_peak else None,
            "frac_of_mma_issue_rate": (achieved / mma_issue) if mma_issue else None,
            "mma_issue_rate": mma_issue,
            "hbm": {"algorithmic_bytes_per_launch": hbm_bytes, "peak_gbs": hbm_peak,
                    "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if
                    peaks.get("hbm_gbs") else "fallback 6.65 TB/s",
                    "achieved_gbs": hbm_bytes / (tensor_ms * 1e-3) / 1e9,
                    "frac": hbm_ms / tensor_ms, "time_at_peak_ms": hbm_ms},
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch "
                              "on the 16-angle profiling case, scaled by angles "
                              "(profiles/k_split_gemm_i8_dense521s.md)" if traffic else None,
            "note": "ops per launch = slice pairs x 8*nangles*N^3 (complex N^3 as a real "
                    "(nangles*N) x 2N x 2N product per slice pair); stage_product_ms adds "
                    "the slicing and exponent kernels of the same stage; ncu of the kernel: "
                    "tensor pipe active 43 %, issue stalls led by long-scoreboard (the "
                    "epilogue's FP64 state loads) and barrier (the accumulator hand-off)"}
    # where the device time of one solve goes (the profiled solve; events between
    # launches make it slightly longer than an unprofiled one)
    breakdown = {"solve_ms": stp["device_ms"], "stage_products_ms": stp["stage_kernel_ms"],
                 "renormalisations_ms": stp["renorm_ms"],
                 "renormalisations": stp["renormalisations"],
                 "rest_ms": stp["device_ms"] - stp["stage_kernel_ms"] - stp["renorm_ms"],
                 "note": "rest = stage-matrix gathers, boundary transforms, intensities"}

    # ---- comparison forms on the same resident problem
    def compare(p):
        solve_ms(p)
        st = solve_ms(p)
        _, f2_ref = rp.fetch()
        return st, f2_ref

    def errors(got, ref):
        rowmax = np.maximum(np.abs(ref).max(axis=1, keepdims=True), 1e-300)
        d = np.abs(got - ref)
        m = np.abs(ref)
        big = m >= 1e-3 * rowmax
        every = np.where(m > 0, d / np.where(m > 0, m, 1.0), np.where(d > 0, np.inf, 0.0))
        return {"max_rel_err_all_spots": float(every.max()),
                "max_err_vs_rowmax": float((d / rowmax).max()),
                "max_rel_err_spots_ge_1e-3_rowmax":
                    float((d / np.where(big, np.abs(ref), np.inf)).max())}

    fp64 = None
    f2_64 = None
    if split and not args.no_fp64:
        # the warm-up solve is profiled (per-launch events of the FP64 stage kernel),
        # the second one is timed without events
        ctx.set_option(native.OPT_PROFILE, 1)
        st64p = solve_ms(native.FP64)
        ctx.set_option(native.OPT_PROFILE, 0)
        st = solve_ms(native.FP64)
        _, f2_64 = rp.fetch()
        fp64 = {"value": nang / (st["device_ms"] / 1e3), "ms_per_step": st["device_ms"],
                "split_speedup": (st["device_ms"] / ms_per_step),
                "roofline": fp64_roofline(st64p, nang, n, f64_peak, peaks,
                                          NCU_TRAFFIC.get((args.workload, "fp64", 0))),
                "breakdown": {"solve_ms": st64p["device_ms"],
                              "stage_products_ms": st64p["stage_kernel_ms"],
                              "renormalisations_ms": st64p["renorm_ms"],
                              "renormalisations": st64p["renormalisations"]}}
        fp64.update({"split_" + k: v for k, v in errors(f2_main, f2_64).items()})
    bf16 = None
    if prec == native.SPLIT_INT8 and not args.no_bf16:
        st, f2_b = compare(native.SPLIT_BF16)
        bf16 = {"value": nang / (st["device_ms"] / 1e3), "ms_per_step": st["device_ms"]}
        if f2_64 is not None:
            bf16.update(errors(f2_b, f2_64))

    # ---- end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        h2d = h2d_bytes(sp, rp)
        t0 = time.perf_counter()
        ang, f2 = sp.srfref(prec)
        first = time.perf_counter() - t0
        t0 = time.perf_counter()
        for _ in range(max(1, args.steps // 2)):
            sp.srfref(prec)
        e_s = (time.perf_counter() - t0) / max(1, args.steps // 2)
        e2e = {"value": nang * ws / e_s, "unit": "angle-solves/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": int(f2.nbytes), "seconds_per_step": e_s,
               "first_call_seconds": first}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        b = cpu_baseline(workdir, s, nang)
        ns = rp.ns
        cpu_value = b["angles"] / (b["seconds"] * ns / b["slices"])
        cpu = {"value": cpu_value, "unit": "angle-solves/s", "cores": b["cores"], "kind": "port",
               "sample": f"median of {len(b['samples_s'])} samples of {b['angles']} angles x "
                         f"first {b['slices']} of {ns} slices on {b['cores']} threads, scaled "
                         "by slice count",
               "samples_s": b["samples_s"], "cpu_model": cpu_model(), "nproc": os.cpu_count()}

    rp.close()
    sp.close()
    uneven = None
    if rank == 0 and ws == 1 and not args.no_uneven:
        uneven = uneven_leg(ctx, prec, per_n=args.uneven_per_n)
    bulk = None
    if rank == 0 and ws == 1 and not args.no_bulk:
        bulk = bulk_leg(ctx, cpu=not args.no_cpu_baseline)
    rk4 = None
    if rank == 0 and ws == 1 and not args.no_rk4:
        rk4 = rk4_leg(ctx)
    ctx.close()

    serve = None
    if rank == 0 and ws == 1 and not args.no_serve:
        serve = {"split" if split else "fp64":
                 serve_leg(local, args.serve_seconds, args.serve_load, prec)}
        if not args.no_serve_fp64 and prec != native.FP64:
            serve["fp64"] = serve_leg(local, args.serve_seconds, args.serve_load, native.FP64)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "angle-solves/s", "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": {native.SPLIT_INT8: f"i8x{slices}-split/f64",
                          native.SPLIT_BF16: f"bf16x{slices}-split/f64", native.FP64: "f64"}[prec],
                "data": "synthetic",
                "config": {"workload": desc, "nb": n, "nangles": nang, "slices": rp.ns,
                           "precision": {native.SPLIT_INT8: "split-int8",
                                         native.SPLIT_BF16: "split-bf16",
                                         native.FP64: "fp64"}[prec],
                           "split_slices": slices if split else None,
                           "renormalisation": "growth bound ln(1e3)",
                           "renormalisations_per_solve": stp["renormalisations"],
                           "stage_products_per_solve": stp["stage_products"],
                           "bulk_boundary": "non-reflecting bulk records (f = 0)",
                           "l2": "inputs larger than L2 (state + stage table > 1 GB)",
                           "parallelism": f"replicas x{ws}",
                           "serving_stream": None if not serve else (
                               f"Poisson {next(iter(serve.values()))['arrival_rate_req_s']:.2f} "
                               f"req/s for {args.serve_seconds:g} s: the serving workload's "
                               "200 req/s scaled to {:g} of the throughput its isolated solve "
                               "times allow".format(args.serve_load))},
                "roofline": roof,
                "e2e": e2e,
                "cpu_baseline": cpu,
                "gpu_launches": launches, "clocks": clk, "wall_seconds_timed": t_wall,
                "serving": serve, "uneven_batch": uneven, "bulk_boundary": bulk,
                "rk4_methods": rk4,
                "breakdown": breakdown,
                "bf16_split": bf16, "fp64": fp64,
                # last, so that a truncated view of the line still shows them
                "split_vs_fp64": None if not fp64 else {
                    "speedup": fp64["split_speedup"],
                    "max_rel_err_all_spots": fp64["split_max_rel_err_all_spots"],
                    "every_spot_within_1e-6": bool(fp64["split_max_rel_err_all_spots"] <= 1e-6),
                    "fp64_value": fp64["value"], "split_value": value,
                    "renormalisation": "growth bound ln(1e3) for both forms; Gauss-Jordan "
                                       "panels of 16 columns (row-per-thread panel kernel) "
                                       "with the trailing update on the FP64 tensor path in "
                                       "both forms; panel arithmetic with fused complex "
                                       "multiply-adds (split) or products formed first (FP64)"}}
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def fp64_roofline(stp: dict, nang: int, n: int, f64_peak, peaks: dict, traffic) -> dict:
    """Roofline of k_stage_gemm_f64 from one profiled FP64 solve: FP64 tensor work
    8*nang*N^3 per launch (complex N^3 per angle) against cuBLAS DGEMM measured in
    the run, and the algorithmic HBM bytes (Q, P read; P, Q' written) against
    MEASURED_PEAKS.json hbm_gbs."""
    nprod = max(stp["stage_products"], 1)
    ms = stp["tensor_kernel_ms"] / nprod
    flop = 8.0 * nang * n ** 3
    achieved = flop / (ms * 1e-3) / 1e12
    peak = f64_peak["sustained"] if f64_peak else None
    hbm_bytes = 4 * 16.0 * nang * n * n
    hbm_peak = peaks.get("hbm_gbs") or 6650.0
    hbm_ms = hbm_bytes / (hbm_peak * 1e9) * 1e3
    flop_ms = flop / (peak * 1e12) * 1e3 if peak else 0.0
    return {"bound": "tensor" if flop_ms >= hbm_ms else "hbm", "achieved": achieved,
            "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
            "traffic": traffic * nang / 16.0 if traffic else None,
            "kernel": "k_stage_gemm_f64 (FP64 DMMA mma.sync.m16n8k4)",
            "peak_source": "cuBLAS DGEMM 8192^3 measured in this run, sustained over a 3 s loop",
            "avg_launch_ms": ms,
            "hbm": {"algorithmic_bytes_per_launch": hbm_bytes, "peak_gbs": hbm_peak,
                    "achieved_gbs": hbm_bytes / (ms * 1e-3) / 1e9, "frac": hbm_ms / ms,
                    "time_at_peak_ms": hbm_ms},
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch "
                              "on the 16-angle profiling case, scaled by angles "
                              "(profiles/k_stage_gemm_f64_dense521s.md)" if traffic else None}


def surface_slices(workdir: Path, s) -> int:
    from oracle import oracle as O
    S = O.Surface(workdir / "bulkP.b", workdir / "surf.txt", s.surface_dz, s.int_method)
    ns = S.ns
    S.close()
    return ns


def h2d_bytes(sp, rp) -> int:
    """Bytes trhepd_srfref copies host->device per call: the mod_scpot3 arrays, the
    stage depths, the beam-pair map and the per-angle gammas, energies and bulk f."""
    p = sp.pot
    natm = p.natms + p.natmb
    b = 8 * (p.nv * 6 * p.nelm + 6 * p.nelm + p.nelm + p.nv)        # asf, b, dchg, Ghk
    b += 8 * 2 * (p.natms + 2 * p.natmb) + 4 * (p.natms + 2 * p.natmb)  # z, ocr, ielm per part
    b += 16 * (p.nv * p.natms + 2 * p.nvb * p.natmb)                 # st0, st1, st2
    b += 8 * rp.ncol + 4 * rp.nb * rp.nb                             # depths, pair map
    ld = -(-rp.nb // 16) * 16
    b += rp.nangles * (16 * rp.nb + 16 * ld + 16 * rp.nb * rp.nb + 8)  # gam, D, F, w
    del natm
    return int(b)


if __name__ == "__main__":
    main()
