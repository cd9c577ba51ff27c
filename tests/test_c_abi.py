"""The C-ABI library loads and exports every entry point include/mvgpu.h declares.

Runs without a GPU: no compute calls, only loading, symbol lookup and the
device-free entry points.
"""
import ctypes as C
import os
import re

import pytest

from meshless_voro_b200 import _native as N
from meshless_voro_b200 import build as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "mvgpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mv_[a-z_0-9]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    B.build()
    return N.lib()


def test_header_symbols_match_binding():
    assert declared_symbols() == sorted(N.EXPORTED)


def test_every_declared_symbol_is_exported(lib):
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_strerror_and_version(lib):
    for code in range(0, 9):
        assert lib.mv_strerror(code)
    assert b"sm_100a" in lib.mv_version()


def test_options_default(lib):
    o = N.Options()
    lib.mv_options_default(C.byref(o))
    assert o.precision == N.MV_PRECISION_FILTERED
    assert o.face_mode == N.MV_FACES_OWNED


def test_shift_from_code(lib):
    w = (C.c_double * 3)(2.0, 3.0, 5.0)
    out = (C.c_double * 3)()
    # m = (1, -1, 0): shift = (w0, -w1, -0.0)
    code = (1 + 1) + 3 * (-1 + 1) + 9 * (0 + 1)
    lib.mv_shift_from_code(code, w, out)
    assert list(out) == [2.0, -3.0, 0.0]
    assert str(out[2]) == "-0.0"


def test_library_built_for_sm100a():
    assert "arch=compute_100a,code=sm_100a" in " ".join(B.NVCC_FLAGS)
    assert "--fmad=false" in B.NVCC_FLAGS


def test_no_device_is_reported_not_faked(lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    h = C.c_void_p()
    assert lib.mv_context_create(-1, C.byref(h)) == N.MV_ERR_NO_DEVICE
