"""Build recipe for libptb200.so (sm_100a).

Each translation unit is compiled by nvcc for ``sm_100a`` only and linked
in-tree into ``particle_transport_b200/libptb200.so``.  ``push_exact.cu``,
``lagstats.cu`` and ``init.cu`` are compiled with ``--fmad=false`` so that
the FP64 parity push, the mu reconstruction (also inside the fused
phase-space binning), the statistics and the particle initialisation keep
the reference's rounding (no fused multiply-add; explicit ``fma`` calls
stay); the other units keep FMA contraction on.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libptb200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", INCLUDE, *ARCH]
UNITS = {
    "push_exact.cu": ["--fmad=false"],
    "init.cu": ["--fmad=false"],
    "push_fast.cu": [],
    "lagstats.cu": ["--fmad=false"],
    "pt_api.cu": [],
    "pt_batch.cu": [],
    "hostio.cu": [],
}


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(out: str, deps) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in ("pt_internal.cuh", "exact_mu.cuh")] + [os.path.join(INCLUDE, "ptb200.h")]
    objs = []
    for unit, flags in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [src, *headers, __file__]):
            cmd = [nvcc(), *COMMON, *flags, *extra, "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    print(build(force="--force" in sys.argv, verbose=True, extra=extra))
