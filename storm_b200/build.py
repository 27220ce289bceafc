"""Build recipe of the FVT step library (libstorm_fvt.so), in-tree, for sm_100a.

Device code is compiled with --fmad=false and host code with -ffp-contract=off so
that every FP64 expression rounds exactly as written, matching the reference's
evaluation order (the oracle uses the same rule).  The FP32 (mixed-precision)
instantiations of the stage kernels (fvt_kernels_f32.cu) are the one exception:
that path is compared with FP64 at a stated tolerance, not bit for bit, so it is
compiled separately with FMA contraction allowed.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libstorm_fvt.so")
SOURCES = ["api.cu", "fvt_kernels.cu", "layout.cpp", "tiles.cpp", "mesh_build.cpp", "noalloc.cu", "gnn_kernels.cu"]
F32_SOURCE = "fvt_kernels_f32.cu"  # includes fvt_kernels.cu
HEADERS = ["fvt_device.cuh", "storm_internal.h", "umma.cuh", os.path.join("..", "..", "include", "storm_fvt.h"),
           os.path.join("..", "..", "include", "storm_gnn.h")]

NVCC_FLAGS = [
    "-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
    "--fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
    "-Xptxas", "-warn-spills",
]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS + [F32_SOURCE]] + [__file__]
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return LIB
    srcs = [os.path.join(CSRC, f) for f in SOURCES]
    f32_obj = LIB + ".f32.o"
    f32_flags = [f for f in NVCC_FLAGS if f != "--fmad=false"] + ["--fmad=true"]
    cmds = [[nvcc(), *f32_flags, "-c", "-o", f32_obj, os.path.join(CSRC, F32_SOURCE)],
            [nvcc(), *NVCC_FLAGS, "-shared", "-o", LIB + ".tmp", *srcs, f32_obj, "-lcudart"]]
    for cmd in cmds:
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed ({r.returncode}):\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr, file=sys.stderr)
    os.replace(LIB + ".tmp", LIB)
    os.remove(f32_obj)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
