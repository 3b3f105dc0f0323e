"""libmbc.so loads and exports every entry point include/mbc.h declares."""
import ctypes as C
import os
import re

import numpy as np

import fastmbcui_b200 as F
from fastmbcui_b200 import _lib

HDR = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "mbc.h")


def declared():
    src = open(HDR).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mbc_[A-Za-z0-9_]+)\s*\(", src)))


def test_header_symbols_exported():
    L = F.load()
    names = declared()
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), n
        assert n in _lib.SIGNATURES, n


def test_status_strings_and_version():
    L = F.load()
    assert L.mbc_status_string(0) == b"ok"
    assert L.mbc_status_string(4) == b"bad argument"
    assert L.mbc_version() >= 100


def test_null_and_bad_arguments_return_status():
    L = F.load()
    h = C.c_void_p()
    assert L.mbc_plan_create(0, None, None, C.byref(h)) == _lib.MBC_BAD_ARG
    assert L.mbc_plan_get_info(None, None) == _lib.MBC_BAD_ARG
    assert L.mbc_solver_create(None, None, 0, None, C.byref(h)) == _lib.MBC_BAD_ARG
    assert L.mbc_solve(None, 1, None, 0, None, 0, None, None, None, None, None) == _lib.MBC_BAD_ARG
    assert L.mbc_minvf_float(None, None, 1, 1, None, 1, None, 1.0, 10, 1e-3, 0, 0, None, None) == _lib.MBC_BAD_ARG
    assert b"NULL" in L.mbc_last_error() or L.mbc_last_error()


def test_context_lifecycle_without_gpu():
    L = F.load()
    h = C.c_void_p()
    assert L.mbc_context_create(C.byref(h)) == 0
    pts = np.zeros((4, 3), np.float32)
    out = C.c_void_p(1)
    # the adjoint before any forward is refused, as in the reference
    s = L.mbc_vpl_fast_float(h, C.c_void_p(8), 4, 4, C.c_void_p(8), 1, pts.ctypes.data, 3.0, 10, 1e-3, 0, 0,
                             out, None)
    assert s == _lib.MBC_BAD_ARG
    assert b"MinvF_float first" in L.mbc_last_error()
    assert L.mbc_context_destroy(h) == 0
