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


def test_default_options_set_every_field():
    """mbc_solve_default_options writes every field of mbc_solve_options, so a
    C caller's struct on the stack holds no garbage afterwards (fp64_recursion,
    the newest field, included)."""
    import ctypes as C

    from fastmbcui_b200 import _lib, load

    o = _lib.SolveOptions()
    C.memset(C.byref(o), 0xFF, C.sizeof(o))
    load().mbc_solve_default_options(C.byref(o))
    want = {"max_iters": 1000, "tol": 1e-8, "schedule": 0, "precondition": 1, "max_refine": 64,
            "inner_tol": 1e-2, "check_every": 8, "true_residual": 0, "profile": 0, "graph": 0, "compact": 0,
            "fp64_recursion": 0}
    assert {k for k, _ in _lib.SolveOptions._fields_} == set(want)
    for k, v in want.items():
        assert getattr(o, k) == v, k


def test_struct_layouts_match_header(tmp_path):
    """The ctypes mirrors of the header's structs have the header's field
    order, offsets and sizes (a C program built against include/mbc.h prints
    them)."""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        import pytest

        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    mirrors = {"mbc_plan_options": _lib.PlanOptions, "mbc_plan_info": _lib.PlanInfo,
               "mbc_operator": _lib.Operator, "mbc_solve_options": _lib.SolveOptions,
               "mbc_solve_stats": _lib.SolveStats, "mbc_factor_tiles": _lib.FactorTiles}
    cfield = {"lambda_": "lambda"}  # Python keywords carry a trailing underscore in the mirrors
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "mbc.h"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'  printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {cfield.get(f, f)}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c99", "-I", os.path.join(root, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln:
            name, field, val = ln.split()
            got[(name, field)] = int(val)
    for cname, py in mirrors.items():
        assert got[(cname, "sizeof")] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)
