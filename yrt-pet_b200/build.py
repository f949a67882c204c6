"""Builds libyrtb.so (the sm_100a kernels + C ABI) in-tree with nvcc.

    python yrt-pet_b200/build.py

The library lands in yrt-pet_b200/lib/ and is what pyyrtpet_b200 loads.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc", "yrtb.cu")
OUT = os.path.join(HERE, "lib", "libyrtb.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

# -fmad=false: the FP32 "mirror" arithmetic must not be contracted into FMAs
# so that it rounds exactly like the reference CPU projector.
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3",
         "-fmad=false", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
         "-I" + os.path.join(ROOT, "include")]


def build(verbose: bool = False) -> str:
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    deps = [SRC, os.path.join(HERE, "csrc", "device.cuh"),
            os.path.join(ROOT, "include", "yrt_b200.h")]
    if os.path.exists(OUT) and all(os.path.getmtime(OUT) >= os.path.getmtime(d)
                                   for d in deps):
        return OUT
    cmd = [NVCC, *FLAGS, SRC, "-o", OUT]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
