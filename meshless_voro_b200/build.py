"""Build recipe of the CUDA library ``libmvgpu.so`` (sm_100a).

The library is built in-tree into ``meshless_voro_b200/_lib/`` so it travels with the
source tree.  f64 code is compiled without FMA contraction (``--fmad=false``) and
with IEEE division and square root, which keeps every f64 value equal to the
reference crate's.  Each source file compiles to its own object (in parallel, into
``_lib/obj``); nvcc then links them into the shared library.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB_DIR = os.path.join(HERE, "_lib")
OBJ_DIR = os.path.join(LIB_DIR, "obj")
LIB = os.path.join(LIB_DIR, "libmvgpu.so")

SOURCES = ["mv_api.cu", "mv_cells.cu", "mv_grid.cu", "mv_noalloc.cu", "mv_staged.cu", "mv_export.cu",
           "mv_tuning.cu"]
HEADERS = ["mv_geom.cuh", "mv_exact.cuh", "mv_internal.h", "mv_cell_common.cuh", "mv_tuning_table.h"]

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    *ARCH,
    "-O3", "-lineinfo", "-std=c++17",
    "--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
]
LINK_FLAGS = [*ARCH, "-shared", "-cudart", "shared"]


def _inputs():
    files = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    files.append(os.path.join(INCLUDE, "mvgpu.h"))
    files.append(os.path.abspath(__file__))
    return files


def is_stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in _inputs())


def _compile(src: str, extra, verbose: bool) -> str:
    obj = os.path.join(OBJ_DIR, os.path.splitext(src)[0] + f".{os.getpid()}.o")
    cmd = [NVCC, *NVCC_FLAGS, *(extra or []), "-I", INCLUDE, "-c", os.path.join(CSRC, src),
           "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return obj


def build(force: bool = False, verbose: bool = False, extra_flags=None) -> str:
    """Compile libmvgpu.so for sm_100a if it is missing or stale; return its path."""
    if not force and not is_stale():
        return LIB
    os.makedirs(OBJ_DIR, exist_ok=True)
    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra_flags, verbose), SOURCES))
    tmp = LIB + f".tmp{os.getpid()}"
    cmd = [NVCC, *LINK_FLAGS, *objs, "-o", tmp]
    if verbose:
        print(" ".join(cmd), flush=True)
    try:
        subprocess.run(cmd, check=True)
    finally:
        for o in objs:
            if os.path.exists(o):
                os.remove(o)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    extra = [a for a in sys.argv[1:] if a.startswith("-X") or a.startswith("--")]
    extra = [a for a in extra if a != "--force"]
    print(build(force="--force" in sys.argv, verbose=True, extra_flags=extra))
