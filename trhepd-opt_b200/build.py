"""Build the sm_100a shared library in-tree: trhepd-opt_b200/_lib/libtrhepd_b200.so.

nvcc cross-compiles for sm_100a without a GPU; the library travels with the
source tree.  Usage: python trhepd-opt_b200/build.py [--verbose]
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "_lib" / "libtrhepd_b200.so"
SOURCES = ["kernels_f64.cu", "split_gemm.cu", "bulk.cu", "magnus.cu", "small.cu", "solver.cu",
           "curves.cu", "noalloc.cu", "cholqr.cu",
           "host_model.cpp", "bulk_model.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or Path(c).exists()):
            return c
    raise RuntimeError("nvcc not found")


def build(verbose: bool = False, force: bool = False) -> Path:
    srcs = [CSRC / s for s in SOURCES]
    deps = srcs + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [
        HERE.parent / "include" / "trhepd_b200.h", Path(__file__)]
    if not force and OUT.exists() and all(OUT.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return OUT
    OUT.parent.mkdir(parents=True, exist_ok=True)
    objs = []
    for s in srcs:
        o = OUT.parent / (s.name + ".o")
        cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
               "-Xptxas", "-v" if verbose else "-O3", "-c", str(s), "-o", str(o)]
        if s.suffix == ".cpp":
            cmd = [nvcc(), "-Wno-deprecated-gpu-targets", "-O3", "-std=c++17", "-Xcompiler",
                   "-fPIC", "-x", "c++", "-c", str(s),
                   "-o", str(o)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode:
            raise RuntimeError(f"nvcc failed on {s.name}")
        objs.append(str(o))
    cmd = [nvcc(), *ARCH, "-Wno-deprecated-gpu-targets", "-shared", "-o", str(OUT), *objs,
           "-lcuda"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    return OUT


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force="--force" in sys.argv))
