"""Builds libavbd6.so (sm_100a) in-tree with nvcc.

The collision translation unit is compiled with -fmad=false so its float
decisions (SAT axis, clip tests, contact selection) match the CPU oracle's
-ffp-contract=off build operation for operation.  The solver units keep FMA
contraction on.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libavbd6.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-ccbin", "g++"]
UNITS = {
    "collide.cu": ["-fmad=false"],
    "solve.cu": [],
    "api.cu": [],
    "mlp.cu": [],
    "noalloc.cu": [],
    "scene.cu": [],
}


def _nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    return os.path.join(cuda, "bin", "nvcc")


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    srcs_mtime = max(os.path.getmtime(os.path.join(CSRC, f)) for f in os.listdir(CSRC))
    hdr = os.path.join(HERE, "..", "include", "avbd6.h")
    srcs_mtime = max(srcs_mtime, os.path.getmtime(hdr))
    for unit, extra in UNITS.items():
        src = os.path.join(CSRC, unit)
        if not os.path.exists(src):
            continue
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        objs.append(obj)
        if os.path.exists(obj) and os.path.getmtime(obj) >= srcs_mtime and not ptxas_info:
            continue
        cmd = [_nvcc(), *ARCH, *COMMON, *extra, "-c", src, "-o", obj]
        if ptxas_info:
            cmd.insert(1, "-Xptxas=-v")
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    if (not os.path.exists(LIB)) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [_nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
