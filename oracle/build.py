"""Build recipe for the CPU oracle (test infrastructure only).

Compiles ``oracle/pt_oracle.c`` into ``oracle/_build/libptoracle.so`` with
``-ffp-contract=off`` so that no multiply-add is fused: the restatement then
reproduces the reference's Float64 expression trees bit for bit.  OpenMP
threads are used only to time the CPU baseline; results do not depend on the
thread count except for the order of floating-point sums across threads,
exactly as in the reference's ``Threads.@threads`` loops.

The reference itself is Julia, so there is no compiled reference to build
into ``oracle/_ref``.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "pt_oracle.c")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libptoracle.so")

CFLAGS = ["-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared", "-std=c11"]


def build(force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = ["gcc", *CFLAGS, SRC, "-o", LIB, "-lm"]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
