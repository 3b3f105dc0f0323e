"""B200-native MFS solve path (maximin ordering -> KL-Cholesky -> PCG).

Python face of libmbc.so (include/mbc.h).  ``Plan`` is host work and runs
without a GPU; ``Solver`` needs a CUDA device.  ``fastmbcui_b200.mfs_torch``
registers the reference's ``mfs_torch`` operators on top of this.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import (MBC_F32, MBC_F64, MBC_FP64_MATVEC_INT8, MBC_FP64_MATVEC_SIMT, MBC_MATVEC_AUTO,
                   MBC_MATVEC_SIMT, MBC_MATVEC_TENSOR,
                   MBC_OP_DENSE, MBC_OP_POINT_KERNEL, MBC_SCHED_BATCHED, MBC_SCHED_PER_RHS, MBC_SCHED_BLOCK, MbcError,
                   check, ptr)

__all__ = ["Plan", "Solver", "MbcError", "load", "plan_many", "solve_many", "MBC_F32", "MBC_F64",
           "MBC_SCHED_BATCHED",
           "MBC_SCHED_PER_RHS", "MBC_SCHED_BLOCK", "MBC_MATVEC_AUTO", "MBC_MATVEC_SIMT", "MBC_MATVEC_TENSOR",
           "MBC_FP64_MATVEC_SIMT", "MBC_FP64_MATVEC_INT8"]


def load():
    return _lib.load()


class Plan:
    """Ordering, pattern and supernodes of a point set (host C++)."""

    def __init__(self, pts, rho: float = 3.0, lam: float = 1.5, max_super: int = 2048,
                 n_threads: int = 0):
        L = load()
        p = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        o = _lib.PlanOptions()
        L.mbc_plan_default_options(C.byref(o))
        o.rho, o.lambda_, o.max_super, o.n_threads = float(rho), float(lam), int(max_super), int(n_threads)
        h = C.c_void_p()
        check(L.mbc_plan_create(p.shape[0], p.ctypes.data, C.byref(o), C.byref(h)), "mbc_plan_create")
        self._h = h
        self.n = p.shape[0]
        self.info = _lib.PlanInfo()
        L.mbc_plan_get_info(h, C.byref(self.info))

    @property
    def handle(self):
        return self._h

    def __del__(self):
        h = getattr(self, "_h", None)
        L = getattr(_lib, "_lib", None) if _lib is not None else None
        if h and L is not None:
            L.mbc_plan_destroy(h)
            self._h = None

    def order(self):
        P = np.empty(self.n, np.int32)
        s = np.empty(self.n, np.float64)
        check(load().mbc_plan_get_order(self._h, P.ctypes.data, s.ctypes.data), "get_order")
        return P, s

    def pattern(self):
        ptr_ = np.empty(self.n + 1, np.int32)
        ind = np.empty(max(1, self.info.pattern_nnz), np.int32)
        check(load().mbc_plan_get_pattern(self._h, ptr_.ctypes.data, ind.ctypes.data), "get_pattern")
        return ptr_, ind[:self.info.pattern_nnz]

    def supernodes(self):
        sp = np.empty(self.info.n_super + 1, np.int32)
        si = np.empty(self.n, np.int32)
        par = np.empty(self.n, np.int32)
        check(load().mbc_plan_get_supernodes(self._h, sp.ctypes.data, si.ctypes.data, par.ctypes.data),
              "get_supernodes")
        return sp, si, par

    def factor_pattern(self):
        lp = np.empty(self.n + 1, np.int32)
        li = np.empty(max(1, self.info.factor_nnz), np.int32)
        check(load().mbc_plan_get_factor_pattern(self._h, lp.ctypes.data, li.ctypes.data),
              "get_factor_pattern")
        return lp, li[:self.info.factor_nnz]

    def factor_rows(self):
        """Row-wise view of the factor pattern (the preconditioner's gather
        order): rptr[n+1], rcol[nnz] (columns, ascending per row), rmap[nnz]
        (positions in the column-wise lind)."""
        nnz = max(1, self.info.factor_nnz)
        rp = np.empty(self.n + 1, np.int32)
        rc = np.empty(nnz, np.int32)
        rm = np.empty(nnz, np.int32)
        check(load().mbc_plan_get_factor_rows(self._h, rp.ctypes.data, rc.ctypes.data, rm.ctypes.data),
              "get_factor_rows")
        return rp, rc[:self.info.factor_nnz], rm[:self.info.factor_nnz]


def spatial_order(pts) -> np.ndarray:
    """Morton (Z-curve) order of points (n x 3, float32 coordinates):
    order[k] = index of the k-th point along the curve (mbc_spatial_order)."""
    p = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
    out = np.empty(p.shape[0], np.int32)
    check(load().mbc_spatial_order(p.shape[0], p.ctypes.data, 3, out.ctypes.data), "mbc_spatial_order")
    return out


def solve_options(**kw) -> _lib.SolveOptions:
    o = _lib.SolveOptions()
    load().mbc_solve_default_options(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown solve option {k}")
        setattr(o, k, v)
    return o


class Solver:
    """Device factor + PCG for one plan and one operator (torch CUDA tensors).

    Keep the tensors that define the operator alive as long as the solver.
    """

    def __init__(self, plan: Plan, *, M=None, x=None, nx=None, y=None, coef: float = 1.0,
                 precision: int = MBC_F64, stream=None, mesh=None):
        """Operator: a dense M (nf x n float32), the point kernel (x, nx: nf x 3;
        y: n x 3), or mesh=(V, faces, S): the matrix-free mesh collocation
        operator (solid angle of each face seen from each source; V: n_vert x
        3 float, faces: nf x 3 int32, S: n x 3), all CUDA tensors."""
        import torch

        L = load()
        op = _lib.Operator()
        if mesh is not None:
            V, Fc, Sy = mesh
            V, Sy = V.contiguous().float(), Sy.contiguous().float()
            Fc = Fc.contiguous().to(torch.int32)
            op.kind, op.nf, op.n = _lib.MBC_OP_MESH, Fc.shape[0], Sy.shape[0]
            op.V, op.faces, op.n_vert, op.y = V.data_ptr(), Fc.data_ptr(), V.shape[0], Sy.data_ptr()
            op.coef = float(coef)
            self._keep = (V, Fc, Sy)
        elif M is not None:
            assert M.is_cuda and M.dtype == torch.float32 and M.dim() == 2
            M = M.contiguous()
            op.kind, op.nf, op.n, op.M, op.ldm = MBC_OP_DENSE, M.shape[0], M.shape[1], M.data_ptr(), M.shape[1]
            self._keep = (M,)
        else:
            xs = [t.contiguous().float() for t in (x, nx, y)]
            op.kind, op.nf, op.n = MBC_OP_POINT_KERNEL, xs[0].shape[0], xs[2].shape[0]
            op.x, op.nx, op.y = (t.data_ptr() for t in xs)
            op.coef = float(coef)
            self._keep = tuple(xs)
        self.plan = plan
        self.precision = precision
        self.nf, self.n = op.nf, op.n
        self._stream = stream
        h = C.c_void_p()
        check(L.mbc_solver_create(plan.handle, C.byref(op), precision, self._sp(), C.byref(h)),
              "mbc_solver_create")
        self._h = h

    def _sp(self):
        import torch

        s = self._stream if self._stream is not None else torch.cuda.current_stream()
        return C.c_void_p(s.cuda_stream)

    def __del__(self):
        h = getattr(self, "_h", None)
        L = getattr(_lib, "_lib", None) if _lib is not None else None
        if h and L is not None:
            L.mbc_solver_destroy(h)
            self._h = None

    def factor(self):
        check(load().mbc_solver_factor(self._h, self._sp()), "mbc_solver_factor")
        return self

    def set_matvec(self, impl: int):
        """MBC_MATVEC_AUTO / _SIMT / _TENSOR (FP32 point-kernel solvers)."""
        check(load().mbc_solver_set_matvec(self._h, int(impl)), "mbc_solver_set_matvec")
        return self

    def set_fp64_matvec(self, impl):
        """How the FP64 matvecs run (mbc_solver_set_fp64_matvec): "simt"
        (MBC_FP64_MATVEC_SIMT, the default) or "int8" (MBC_FP64_MATVEC_INT8,
        exact digit slicing on the INT8 tensor cores, 10 bytes of device
        memory per matrix entry)."""
        impl = {"simt": MBC_FP64_MATVEC_SIMT, "int8": MBC_FP64_MATVEC_INT8}.get(impl, impl)
        check(load().mbc_solver_set_fp64_matvec(self._h, int(impl)), "mbc_solver_set_fp64_matvec")
        self.fp64_matvec = int(impl)
        return self

    def prepare(self):
        """Build what the selected matvecs need now (mbc_solver_prepare)."""
        check(load().mbc_solver_prepare(self._h, self._sp()), "mbc_solver_prepare")
        return self

    def set_factor_tiles(self, tiles: dict):
        """Factor tile shapes (mbc_solver_set_factor_tiles): {"max_ns": [3],
        "tile_rows": [4], "tc_min_ns": int (optional; absent keeps the
        solver's)}."""
        t = _lib.FactorTiles()
        check(load().mbc_solver_get_factor_tiles(self._h, C.byref(t)), "mbc_solver_get_factor_tiles")
        t.max_ns[:] = [int(v) for v in tiles["max_ns"]]
        t.tile_rows[:] = [int(v) for v in tiles["tile_rows"]]
        if "tc_min_ns" in tiles:
            t.tc_min_ns = int(tiles["tc_min_ns"])
        check(load().mbc_solver_set_factor_tiles(self._h, C.byref(t)), "mbc_solver_set_factor_tiles")
        return self

    def factor_tiles(self) -> dict:
        t = _lib.FactorTiles()
        check(load().mbc_solver_get_factor_tiles(self._h, C.byref(t)), "mbc_solver_get_factor_tiles")
        return t.as_dict()

    def tune_factor(self, reps: int = 2):
        """Autotune the factor's tile shapes on this solver (mbc_solver_tune_factor);
        returns (tiles, best factor ms).  The solver ends factored with them."""
        t = _lib.FactorTiles()
        ms = C.c_double()
        check(load().mbc_solver_tune_factor(self._h, int(reps), C.byref(t), C.byref(ms), self._sp()),
              "mbc_solver_tune_factor")
        return t.as_dict(), ms.value

    def set_wait_limit(self, polls: int):
        """Polls before a tensor-core kernel's wait for a partner gives up
        (mbc_solver_set_wait_limit; 0: the default).  For failure-path tests."""
        check(load().mbc_solver_set_wait_limit(self._h, int(polls)), "mbc_solver_set_wait_limit")
        return self

    def tensor_grams(self) -> int:
        """Supernodes of the last factor whose Gram ran on the tensor cores."""
        c = C.c_int32(0)
        check(load().mbc_solver_get_tensor_grams(self._h, C.byref(c)), "get_tensor_grams")
        return c.value

    def pivot_retries(self) -> int:
        c = C.c_int32(0)
        check(load().mbc_solver_get_pivot_retries(self._h, C.byref(c)), "get_pivot_retries")
        return int(c.value)

    def get_factor(self, theta: bool = False):
        lval = np.empty(max(1, self.plan.info.factor_nnz), np.float64)
        th = np.empty(max(1, self.plan.info.theta_nnz), np.float64) if theta else None
        check(load().mbc_solver_get_factor(self._h, lval.ctypes.data, None if th is None else th.ctypes.data),
              "get_factor")
        return (lval[:self.plan.info.factor_nnz], None if th is None else th[:self.plan.info.theta_nnz])

    def _dt(self, t):
        import torch

        return MBC_F64 if t.dtype == torch.float64 else MBC_F32

    def solve(self, F, X0=None, out_dtype=None, iters=False, ok_not_converged=True, **opts):
        """Forward solve for every column of F (nf x R); returns (X, stats[, iters])."""
        import torch

        F = F.contiguous()
        R = 1 if F.dim() == 1 else F.shape[1]
        dt = out_dtype or F.dtype
        X = torch.empty((self.n, R), dtype=dt, device=F.device)
        if X0 is not None:
            X0 = X0.to(dt).contiguous()
        o = solve_options(**opts)
        st = _lib.SolveStats()
        it = np.zeros(R, np.int32)
        s = load().mbc_solve(self._h, R, F.data_ptr(), self._dt(F), X.data_ptr(), self._dt(X),
                             None if X0 is None else X0.data_ptr(), C.byref(o), C.byref(st),
                             it.ctypes.data, self._sp())
        ok = (_lib.MBC_OK, _lib.MBC_NOT_CONVERGED) if ok_not_converged else (_lib.MBC_OK,)
        check(s, "mbc_solve", ok)
        X = X[:, 0] if F.dim() == 1 else X
        return (X, st.as_dict(), it) if iters else (X, st.as_dict())

    def solve_adjoint(self, B, out_dtype=None, iters=False, ok_not_converged=True, **opts):
        import torch

        B = B.contiguous()
        R = 1 if B.dim() == 1 else B.shape[1]
        dt = out_dtype or B.dtype
        X = torch.empty((self.n, R), dtype=dt, device=B.device)
        o = solve_options(**opts)
        st = _lib.SolveStats()
        it = np.zeros(R, np.int32)
        s = load().mbc_solve_adjoint(self._h, R, B.data_ptr(), self._dt(B), X.data_ptr(), self._dt(X),
                                     C.byref(o), C.byref(st), it.ctypes.data, self._sp())
        ok = (_lib.MBC_OK, _lib.MBC_NOT_CONVERGED) if ok_not_converged else (_lib.MBC_OK,)
        check(s, "mbc_solve_adjoint", ok)
        X = X[:, 0] if B.dim() == 1 else X
        return (X, st.as_dict(), it) if iters else (X, st.as_dict())

    def apply_K(self, V):
        import torch

        V = V.contiguous()
        R = 1 if V.dim() == 1 else V.shape[1]
        W = torch.empty((self.nf, R), dtype=V.dtype, device=V.device)
        check(load().mbc_apply_K(self._h, R, V.data_ptr(), W.data_ptr(), self._sp()), "mbc_apply_K")
        return W[:, 0] if V.dim() == 1 else W

    def apply_KT(self, W):
        import torch

        W = W.contiguous()
        R = 1 if W.dim() == 1 else W.shape[1]
        T = torch.empty((self.n, R), dtype=W.dtype, device=W.device)
        check(load().mbc_apply_KT(self._h, R, W.data_ptr(), T.data_ptr(), self._sp()), "mbc_apply_KT")
        return T[:, 0] if W.dim() == 1 else T

    def added_mass(self, X, weights, body_ptr, centers, rho_fluid=1.0, accel=None):
        """Added-mass tensor (6 bodies x R, FP64) of strengths X (n x R, original
        order) and, given a generalized acceleration (R = 6 bodies), the fluid
        forces -Mf a (mbc_added_mass).  weights: nf quadrature weights."""
        import torch

        X = X.contiguous()
        if X.dim() == 1:
            X = X[:, None]
        R = X.shape[1]
        w = torch.as_tensor(np.asarray(weights, np.float32), device=X.device).contiguous()
        bp = np.ascontiguousarray(body_ptr, np.int32)
        cen = np.ascontiguousarray(centers, np.float64)
        nb = bp.shape[0] - 1
        Mf = np.empty((6 * nb, R), np.float64)
        acc = None if accel is None else np.ascontiguousarray(accel, np.float64)
        frc = None if accel is None else np.empty(6 * nb, np.float64)
        dt = MBC_F64 if X.dtype == torch.float64 else MBC_F32
        check(load().mbc_added_mass(self._h, R, X.data_ptr(), dt, w.data_ptr(), nb, bp.ctypes.data,
                                    cen.ctypes.data, float(rho_fluid), Mf.ctypes.data,
                                    None if acc is None else acc.ctypes.data,
                                    None if frc is None else frc.ctypes.data, self._sp()),
              "mbc_added_mass")
        return (Mf, frc) if accel is not None else Mf


def plan_many(specs, threads=None):
    """Host plans of many scenes at once: specs = [(points, rho, lam,
    max_super), ...], planned on a thread pool (the plan code keeps no shared
    state and the binding releases the interpreter lock during the call).
    The host cores are divided among the pool's plans (each plan's own
    parallel stages get cores / workers threads), so they do not oversubscribe.
    Returns the Plans in input order, identical to planning them one by one."""
    import os
    from concurrent.futures import ThreadPoolExecutor

    specs = list(specs)
    if not specs:
        return []
    cores = os.cpu_count() or 1
    workers = threads or min(len(specs), cores)
    inner = max(1, cores // workers)
    with ThreadPoolExecutor(max_workers=workers) as ex:
        return list(ex.map(lambda a: Plan(*a, n_threads=inner), specs))


def solve_many(solvers, Fs, X0s=None, threads=None, factor=True, **opts):
    """Factor and solve independent scenes concurrently: each solver on its
    own CUDA stream, driven by its own host thread (the library's calls
    release the interpreter lock), so small scenes fill the GPU together.
    Returns [(X, stats)] in input order.  Results are bitwise those of
    solving the scenes one by one: every kernel reduces in a fixed order."""
    import torch
    from concurrent.futures import ThreadPoolExecutor

    dev = torch.cuda.current_device()
    X0s = list(X0s) if X0s is not None else [None] * len(solvers)
    producer = torch.cuda.current_stream()

    def work(i):
        torch.cuda.set_device(dev)
        st = torch.cuda.Stream()
        st.wait_stream(producer)  # the inputs were made on the caller's stream
        with torch.cuda.stream(st):
            if factor:
                solvers[i].factor()
            X, stats = solvers[i].solve(Fs[i], X0=X0s[i], **opts)
        st.synchronize()
        return X, stats

    with ThreadPoolExecutor(max_workers=threads or min(8, max(1, len(solvers)))) as ex:
        return list(ex.map(work, range(len(solvers))))
