"""ctypes binding of include/mbc.h (libmbc.so, built in-tree).

There is no fallback: if libmbc.so is missing or fails to load, importing the
package raises.  Device arrays are passed as raw pointers (torch tensors'
``data_ptr()``), host arrays as numpy buffers.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libmbc.so")

MBC_OK, MBC_NOT_CONVERGED, MBC_BREAKDOWN, MBC_NONSPD_PIVOT, MBC_BAD_ARG = 0, 1, 2, 3, 4
MBC_CUDA_ERROR, MBC_TIMEOUT, MBC_NO_MEMORY, MBC_COVERAGE, MBC_UNSUPPORTED = 5, 6, 7, 8, 9
MBC_F64, MBC_F32 = 0, 1
MBC_OP_DENSE, MBC_OP_POINT_KERNEL, MBC_OP_MESH = 0, 1, 2
MBC_SCHED_BATCHED, MBC_SCHED_PER_RHS, MBC_SCHED_BLOCK = 0, 1, 2
MBC_MATVEC_AUTO, MBC_MATVEC_SIMT, MBC_MATVEC_TENSOR = 0, 1, 2
MBC_FP64_MATVEC_SIMT, MBC_FP64_MATVEC_INT8 = 0, 1


class PlanOptions(C.Structure):
    _fields_ = [("rho", C.c_double), ("lambda_", C.c_double), ("max_super", C.c_int32),
                ("n_threads", C.c_int32)]


class PlanInfo(C.Structure):
    _fields_ = [("n", C.c_int32), ("n_super", C.c_int32), ("pattern_nnz", C.c_int64),
                ("factor_nnz", C.c_int64), ("theta_nnz", C.c_int64), ("max_set", C.c_int32),
                ("root", C.c_int32), ("t_order_ms", C.c_double), ("t_pattern_ms", C.c_double),
                ("t_super_ms", C.c_double)]


class Operator(C.Structure):
    _fields_ = [("kind", C.c_int32), ("nf", C.c_int32), ("n", C.c_int32), ("M", C.c_void_p),
                ("ldm", C.c_int64), ("x", C.c_void_p), ("nx", C.c_void_p), ("y", C.c_void_p),
                ("coef", C.c_double), ("V", C.c_void_p), ("faces", C.c_void_p), ("n_vert", C.c_int32)]


class SolveOptions(C.Structure):
    _fields_ = [("max_iters", C.c_int32), ("tol", C.c_double), ("schedule", C.c_int32),
                ("precondition", C.c_int32), ("max_refine", C.c_int32), ("inner_tol", C.c_double),
                ("check_every", C.c_int32), ("true_residual", C.c_int32), ("profile", C.c_int32),
                ("graph", C.c_int32), ("compact", C.c_int32), ("fp64_recursion", C.c_int32)]


class FactorTiles(C.Structure):
    _fields_ = [("max_ns", C.c_int32 * 3), ("tile_rows", C.c_int32 * 4), ("tc_min_ns", C.c_int32)]

    def as_dict(self):
        return {"max_ns": list(self.max_ns), "tile_rows": list(self.tile_rows), "tc_min_ns": int(self.tc_min_ns)}


class SolveStats(C.Structure):
    _fields_ = [("status_per_worst", C.c_int32), ("iters_max", C.c_int32),
                ("iters_total", C.c_int64), ("refinements", C.c_int32),
                ("n_converged", C.c_int32), ("relres_max", C.c_double),
                ("true_relres_max", C.c_double), ("t_solve_ms", C.c_double),
                ("t_matvec_ms", C.c_double), ("n_matvec", C.c_int64), ("kernel_launches", C.c_int64),
                ("n_polished", C.c_int32), ("t_matvec64_ms", C.c_double), ("n_matvec64", C.c_int64),
                ("matvec64_columns", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# every entry point declared in include/mbc.h: name -> (restype, argtypes)
_vp, _i32, _i64, _d = C.c_void_p, C.c_int32, C.c_int64, C.c_double
SIGNATURES = {
    "mbc_status_string": (C.c_char_p, [C.c_int]),
    "mbc_last_error": (C.c_char_p, []),
    "mbc_version": (C.c_int32, []),
    "mbc_plan_default_options": (None, [C.POINTER(PlanOptions)]),
    "mbc_plan_create": (C.c_int, [_i32, _vp, C.POINTER(PlanOptions), C.POINTER(_vp)]),
    "mbc_plan_destroy": (C.c_int, [_vp]),
    "mbc_plan_get_info": (C.c_int, [_vp, C.POINTER(PlanInfo)]),
    "mbc_plan_get_order": (C.c_int, [_vp, _vp, _vp]),
    "mbc_plan_get_pattern": (C.c_int, [_vp, _vp, _vp]),
    "mbc_plan_get_supernodes": (C.c_int, [_vp, _vp, _vp, _vp]),
    "mbc_plan_get_factor_pattern": (C.c_int, [_vp, _vp, _vp]),
    "mbc_spatial_order": (C.c_int, [_i32, _vp, _i32, _vp]),
    "mbc_minvf_grad": (C.c_int, [_i32, _i32, _i32, _vp, _i64, _vp, _vp, _vp, _vp, _vp, _i64, _vp, _vp]),
    "mbc_factor_default_tiles": (None, [C.POINTER(FactorTiles)]),
    "mbc_solver_set_factor_tiles": (C.c_int, [_vp, C.POINTER(FactorTiles)]),
    "mbc_solver_get_factor_tiles": (C.c_int, [_vp, C.POINTER(FactorTiles)]),
    "mbc_solver_tune_factor": (C.c_int, [_vp, _i32, C.POINTER(FactorTiles), C.POINTER(C.c_double), _vp]),
    "mbc_solver_get_tensor_grams": (C.c_int, [_vp, C.POINTER(C.c_int32)]),
    "mbc_solver_set_wait_limit": (C.c_int, [_vp, C.c_uint32]),
    "mbc_plan_get_factor_rows": (C.c_int, [_vp, _vp, _vp, _vp]),
    "mbc_solver_create": (C.c_int, [_vp, C.POINTER(Operator), _i32, _vp, C.POINTER(_vp)]),
    "mbc_solver_destroy": (C.c_int, [_vp]),
    "mbc_solver_factor": (C.c_int, [_vp, _vp]),
    "mbc_solver_get_factor": (C.c_int, [_vp, _vp, _vp]),
    "mbc_solver_get_pivot_retries": (C.c_int, [_vp, C.POINTER(_i32)]),
    "mbc_solver_set_matvec": (C.c_int, [_vp, _i32]),
    "mbc_solver_set_fp64_matvec": (C.c_int, [_vp, _i32]),
    "mbc_solver_prepare": (C.c_int, [_vp, _vp]),
    "mbc_solve_default_options": (None, [C.POINTER(SolveOptions)]),
    "mbc_solve": (C.c_int, [_vp, _i32, _vp, _i32, _vp, _i32, _vp, C.POINTER(SolveOptions),
                            C.POINTER(SolveStats), _vp, _vp]),
    "mbc_solve_adjoint": (C.c_int, [_vp, _i32, _vp, _i32, _vp, _i32, C.POINTER(SolveOptions),
                                    C.POINTER(SolveStats), _vp, _vp]),
    "mbc_apply_K": (C.c_int, [_vp, _i32, _vp, _vp, _vp]),
    "mbc_apply_KT": (C.c_int, [_vp, _i32, _vp, _vp, _vp]),
    "mbc_added_mass": (C.c_int, [_vp, _i32, _vp, _i32, _vp, _i32, _vp, _vp, _d, _vp, _vp, _vp, _vp]),
    "mbc_mlp_create": (C.c_int, [_i32, _i32, _i32, _i32, C.c_uint64, C.POINTER(_vp)]),
    "mbc_mlp_destroy": (C.c_int, [_vp]),
    "mbc_mlp_num_params": (C.c_int, [_vp, C.POINTER(_i64)]),
    "mbc_mlp_get_params": (C.c_int, [_vp, _vp]),
    "mbc_mlp_set_params": (C.c_int, [_vp, _vp]),
    "mbc_mlp_forward": (C.c_int, [_vp, _i32, _vp, _vp, _vp]),
    "mbc_mlp_train_step": (C.c_int, [_vp, _i32, _vp, _vp, C.c_float, _vp, _vp, _vp]),
    "mbc_warm_correct": (C.c_int, [_i32, _i32, _vp, _i32, _vp, _vp, _vp, _vp]),
    "mbc_mesh_assemble": (C.c_int, [_i32, _vp, _i32, _vp, _vp, _i32, _vp, _i32, _vp, _i32, _vp, _i64, _vp,
                                    _vp]),
    "mbc_point_apply_noalloc": (C.c_int, [_i32, _i32, _i32, _vp, _vp, _vp, C.c_double, _i32, _vp, _vp, _vp]),
    "mbc_context_create": (C.c_int, [C.POINTER(_vp)]),
    "mbc_context_destroy": (C.c_int, [_vp]),
    "mbc_context_last_stats": (C.c_int, [_vp, C.POINTER(SolveStats)]),
    "mbc_minvf_float": (C.c_int, [_vp, _vp, _i32, _i32, _vp, _i32, _vp, _d, _i64, _d, _i32, _i32,
                                  _vp, _vp]),
    "mbc_vpl_fast_float": (C.c_int, [_vp, _vp, _i32, _i32, _vp, _i32, _vp, _d, _i64, _d, _i32,
                                     _i32, _vp, _vp]),
}

_lib = None


class MbcError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = _lib.mbc_last_error().decode() if _lib is not None else ""
        name = _lib.mbc_status_string(status).decode() if _lib is not None else str(status)
        super().__init__(f"{where}: {name} ({status}): {msg}")
        self.status = status


def load():
    """Load libmbc.so (raises OSError when it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: build it with `python -m fastmbcui_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int, where: str, ok=(MBC_OK,)):
    if status not in ok:
        raise MbcError(status, where)
    return status


def ptr(a) -> int:
    """Raw pointer of a numpy array or torch tensor."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()
