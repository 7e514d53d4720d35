"""Build libquill_b200.so (sm_100a) in-tree with nvcc.

    python -m quill_b200.build          # incremental
    python -m quill_b200.build --force  # rebuild everything

The FP64 kernels are compiled with --fmad=false so that their arithmetic is
the plain IEEE operation sequence of the reference; the mixed-precision and
integer kernels keep fused multiply-adds.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libquill_b200.so")
DRIVER = os.path.join(PKG, "qp_driver")
DRIVER_SRC = os.path.join(PKG, "driver", "qp_driver.cpp")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "--expt-relaxed-constexpr", f"-I{os.path.join(ROOT, 'include')}"]

# (source, extra flags)
SOURCES = [
    ("qp_fp64.cu", ["--fmad=false"]),
    # FP32 path: approximate division / square root (within 2 ulp), denormals flushed
    ("qp_mixed.cu", ["--prec-div=false", "--prec-sqrt=false", "--ftz=true"]),
    ("qp_rebin.cu", []),
    ("qp_load.cu", []),
    ("qp_noalloc.cu", []),
    ("qp_adjoint.cu", ["--fmad=false"]),
    ("qp_ordered.cu", ["--fmad=false"]),
    ("qp_merge.cu", []),
    ("qp_window.cu", []),
    ("qp_catch.cu", []),
    ("qp_track.cu", []),
    ("qp_slab.cu", []),
    ("qp_api.cu", []),
]
# every header of csrc/ is a dependency of every translation unit
HEADERS = sorted(f for f in os.listdir(CSRC) if f.endswith((".h", ".cuh")))


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "quill_b200.h")]
    objs = []
    for src, extra in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _newer(o, [s] + hdrs + [__file__]):
            cmd = [NVCC] + ARCH + COMMON + extra + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _newer(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if force or _newer(DRIVER, [DRIVER_SRC, LIB, os.path.join(ROOT, "include", "quill_b200.h")]):
        cmd = ["g++", "-O2", "-std=c++17", f"-I{os.path.join(ROOT, 'include')}", DRIVER_SRC, "-o", DRIVER,
               f"-L{PKG}", "-lquill_b200", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
