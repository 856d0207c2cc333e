"""Per-device keying of the shared-memory opt-in (csrc/launch_attr.h), on the CPU:
the header is compiled with g++ against a stand-in of the two CUDA runtime calls
it makes, which records every attribute call and lets the test switch devices."""
from __future__ import annotations

import subprocess
import textwrap

from conftest import ROOT

FAKE_RUNTIME = textwrap.dedent("""
    #pragma once
    #include <cstddef>
    typedef int cudaError_t;
    enum { cudaSuccess = 0 };
    enum cudaFuncAttribute { cudaFuncAttributeMaxDynamicSharedMemorySize = 8 };
    extern int g_device, g_calls[4], g_last[4];
    inline cudaError_t cudaGetDevice(int* d) { *d = g_device; return cudaSuccess; }
    inline cudaError_t cudaFuncSetAttribute(const void*, cudaFuncAttribute, int v) {
      g_calls[g_device]++; g_last[g_device] = v; return cudaSuccess;
    }
""")

MAIN = textwrap.dedent("""
    #include "launch_attr.h"
    #include <cstdio>
    int g_device = 0, g_calls[4] = {0, 0, 0, 0}, g_last[4] = {0, 0, 0, 0};
    static void kern() {}
    int main() {
      trhepd::SmemOptIn a;
      a.ensure((const void*)kern, 1000);
      a.ensure((const void*)kern, 1000);       // same device, same size: no call
      g_device = 1;
      a.ensure((const void*)kern, 1000);       // another device: its own call
      a.ensure((const void*)kern, 500);        // smaller than set: no call
      g_device = 0;
      a.ensure((const void*)kern, 2000);       // larger: raised
      std::printf("%d %d %d %d %zu %zu\\n", g_calls[0], g_calls[1], g_last[0], g_last[1],
                  a.bytes_on(0), a.bytes_on(1));
      return 0;
    }
""")


def test_smem_opt_in_is_per_device(tmp_path):
    (tmp_path / "cuda_runtime.h").write_text(FAKE_RUNTIME)
    (tmp_path / "main.cpp").write_text(MAIN)
    exe = tmp_path / "t"
    subprocess.run(["g++", "-std=c++17", "-I", str(tmp_path), "-I",
                    str(ROOT / "trhepd-opt_b200" / "csrc"), str(tmp_path / "main.cpp"), "-o",
                    str(exe), "-pthread"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    assert out == ["2", "1", "2000", "1000", "2000", "1000"]
