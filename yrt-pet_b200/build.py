"""Builds libyrtb.so (the sm_100a kernels + C ABI) in-tree with nvcc, and
libyrtb_l2bench.so (the L2 request-throughput measurement the benchmark's
roofline uses).

    python yrt-pet_b200/build.py

The libraries land in yrt-pet_b200/lib/; pyyrtpet_b200 loads libyrtb.so.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc", "yrtb.cu")
OUT = os.path.join(HERE, "lib", "libyrtb.so")
L2_SRC = os.path.join(HERE, "csrc", "l2_bench.cu")
L2_OUT = os.path.join(HERE, "lib", "libyrtb_l2bench.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

# -fmad=false: the FP32 "mirror" arithmetic must not be contracted into FMAs
# so that it rounds exactly like the reference CPU projector.
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3",
         "-fmad=false", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
         "-I" + os.path.join(ROOT, "include")]


def _compile(src, out, deps, verbose):
    if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d)
                                   for d in deps):
        return
    cmd = [NVCC, *FLAGS, src, "-o", out]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)


def build(verbose: bool = False) -> str:
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    _compile(SRC, OUT, [SRC, os.path.join(HERE, "csrc", "device.cuh"),
                        os.path.join(ROOT, "include", "yrt_b200.h")], verbose)
    _compile(L2_SRC, L2_OUT, [L2_SRC], verbose)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
