"""Build liblmmstokes.so in-tree for sm_100a (B200).

    python -m lowmachmixtures_b200.build
    python -m lowmachmixtures_b200.build --bounds-check   # liblmmstokes_bc.so

The bounds-check library is compiled with -DLMM_BOUNDS_CHECK: every stencil
load tests its address against the registered device allocations and a
solve that made an out-of-range load returns LMM_ERR_BOUNDS (stencil.cuh).
Set LMM_BOUNDS_CHECK=1 to make the package load it instead of the default.

The FP64 translation units are compiled with -fmad=false so that every
multiply and add rounds separately in the reference's operand order; the FP32
preconditioner unit keeps FMA contraction.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "liblmmstokes.so")
BUILD_BC = os.path.join(PKG, "_build_bc")
LIB_BC = os.path.join(PKG, "liblmmstokes_bc.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
          "--expt-relaxed-constexpr", "-I" + os.path.join(os.path.dirname(PKG), "include")]

UNITS = [
    ("kernels_fp64.cu", ["-fmad=false"]),
    ("kernels_fp32.cu", ["-fmad=true"]),
    ("walls_fp64.cu", ["-fmad=false"]),
    ("walls_fp32.cu", ["-fmad=true"]),
    ("krylov.cu", ["-fmad=false"]),
    ("solver.cu", ["-fmad=false"]),
    ("noalloc.cu", ["-fmad=false"]),
    ("autotune.cu", []),
    ("nn.cu", ["-fmad=true"]),
    ("net.cu", ["-fmad=true"]),
    ("learned.cu", ["-fmad=true"]),
    ("ensemble.cu", ["-fmad=false"]),
    ("stochastic.cu", ["-fmad=false"]),
]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(src_list, target) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in src_list)


def build(verbose: bool = False, force: bool = False, extra: list | None = None, bounds_check: bool = False) -> str:
    bdir, lib = (BUILD_BC, LIB_BC) if bounds_check else (BUILD, LIB)
    extra = (extra or []) + (["-DLMM_BOUNDS_CHECK"] if bounds_check else [])
    os.makedirs(bdir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(os.path.dirname(PKG), "include", "lmm_stokes.h"))
    objs = []
    cc = nvcc()
    jobs = []
    for src, flags in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(bdir, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale([s] + headers, o):
            cmd = [cc, "-c", s, "-o", o] + ARCH + COMMON + flags + extra
            if verbose:
                print(" ".join(cmd), flush=True)
            jobs.append(cmd)
    # translation units compile in parallel (the instantiation units dominate)
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(subprocess.run, cmd, check=True) for cmd in jobs]:
            f.result()
    if force or _stale(objs, lib):
        cmd = [cc, "-shared", "-o", lib] + objs + ARCH + ["-Xcompiler", "-fPIC"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return lib


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, bounds_check="--bounds-check" in sys.argv)
