"""Builds libpasta_b200.so in-tree for sm_100a (nvcc, no JIT cache).

prep.cu and binary.cu are compiled with -fmad=false so that their
double-precision geometry (neighbour search, kernel widths, windows, swarm
clamps, shifts) is evaluated exactly as written, like the host and the
reference; the bandwidth/FFT kernels keep FMA contraction.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libpasta_b200.so")
ROOT = os.path.dirname(HERE)
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
          "-I" + os.path.join(ROOT, "include")]
UNITS = [("prep.cu", ["-fmad=false"]), ("kernels.cu", []), ("binary.cu", ["-fmad=false"]), ("lintc.cu", []), ("interp_tc.cu", []),
         ("engine.cu", []), ("noalloc.cu", [])]
DEPS = ["common.cuh", "fft.cuh", "kernels.h"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    srcs = [os.path.join(CSRC, u) for u, _ in UNITS] + [os.path.join(CSRC, d) for d in DEPS]
    srcs.append(os.path.join(ROOT, "include", "pasta_b200.h"))
    return any(os.path.getmtime(s) > t for s in srcs)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objs = []
    for unit, extra in UNITS:
        obj = os.path.join(LIBDIR, unit.replace(".cu", ".o"))
        cmd = [_nvcc()] + ARCH + COMMON + extra + ["-c", os.path.join(CSRC, unit), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    subprocess.run([_nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
