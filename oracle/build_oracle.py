"""Build recipe for the CPU oracle (test infrastructure only).

Compiles ``oracle/mv_oracle.cpp`` into ``oracle/_build/libmv_oracle.so`` with IEEE
binary64 semantics (no FMA contraction, no fast-math) and OpenMP.  The Rust reference
cannot be compiled in this image (no cargo/rustc), so there is no ``oracle/_ref``.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "mv_oracle.cpp")
OUT_DIR = os.path.join(HERE, "_build")
OUT = os.path.join(OUT_DIR, "libmv_oracle.so")

CXXFLAGS = [
    "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp",
    "-ffp-contract=off", "-fno-fast-math", "-march=x86-64", "-mtune=generic",
]


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the oracle shared library if it is missing or stale; return its path."""
    if (not force and os.path.exists(OUT)
            and os.path.getmtime(OUT) >= os.path.getmtime(SRC)):
        return OUT
    os.makedirs(OUT_DIR, exist_ok=True)
    tmp = OUT + f".tmp{os.getpid()}"
    cmd = ["g++", *CXXFLAGS, SRC, "-o", tmp]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
