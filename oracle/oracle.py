"""Python face of the CPU ORACLE (test infrastructure only).

Loads oracle/_build/liboracle.so (the FP64 C restatement in mbc_oracle.c)
and, when present, oracle/_ref/libref.so (the reference's own maxmin.h and
nanoflann.hpp, compiled by oracle/Makefile).  Only tests/, the smoke check
and bench.py's CPU-baseline leg import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(HERE, "_build", "liboracle.so")
_REF = os.path.join(HERE, "_ref", "libref.so")

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _vp(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        L.orc_order.argtypes = [C.c_int, _f64p, _i32p, _f64p]
        L.orc_root.argtypes = [C.c_int, _f64p]
        L.orc_pattern.restype = C.c_int64
        L.orc_pattern.argtypes = [C.c_int, _f64p, _f64p, C.c_double, _i32p, C.c_void_p]
        L.orc_aggregate.argtypes = [C.c_int, _i32p, _i32p, _f64p, C.c_double, C.c_int,
                                    _i32p, _i32p, _i32p, _i32p]
        L.orc_super_sets.restype = C.c_int64
        L.orc_super_sets.argtypes = [C.c_int, _i32p, _i32p, C.c_int, _i32p, _i32p, C.c_void_p]
        L.orc_super_pattern.restype = C.c_int64
        L.orc_super_pattern.argtypes = [C.c_int, _i32p, _i32p, _i32p, _i32p, C.c_void_p]
        vp = C.c_void_p
        L.orc_apply_K.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, C.c_double, C.c_int, _f64p, _f64p]
        L.orc_apply_KT.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, C.c_double, C.c_int, _f64p, _f64p]
        L.orc_factor.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, C.c_double, _i32p, C.c_int,
                                 _i32p, _i32p, _i32p, _i32p, _i64p, _f64p, _i32p, _i32p, _f64p,
                                 C.POINTER(C.c_int32)]
        L.orc_mesh_solid_angle.argtypes = [C.c_int, _f64p, _i32p, C.c_int, _f64p, _f64p]
        L.orc_mesh_solid_angle.restype = None
        L.orc_mesh_rhs.argtypes = [C.c_int, _f64p, _i32p, _i32p, C.c_int, _f64p, _f64p]
        L.orc_oz_apply.argtypes = [C.c_int, C.c_int, C.c_int, _f64p, _f64p, C.c_double, _f64p]
        L.orc_mesh_rhs.restype = None
        L.orc_added_mass.argtypes = [C.c_int, C.c_int, _f64p, _f64p, _f64p, C.c_int, _f64p, _f64p, C.c_int,
                                     _i32p, _f64p, C.c_double, _f64p]
        L.orc_added_mass.restype = None
        L.orc_precond.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, _f64p]
        L.orc_pcg.restype = C.c_int
        L.orc_pcg.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, C.c_double, _i32p, _i32p, _i32p,
                              _f64p, C.c_int, vp, vp, C.c_int, C.c_int, C.c_double, _f64p,
                              C.POINTER(C.c_double)]
        L.orc_pcg_many.restype = C.c_int
        L.orc_pcg_many.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, C.c_double, _i32p, _i32p, _i32p,
                                   _f64p, C.c_int, _f64p, C.c_int, C.c_double, _f64p, _i32p, _f64p]
        L.orc_num_threads.restype = C.c_int
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(_REF)


def ref():
    global _ref
    if _ref is None:
        R = C.CDLL(_REF)
        R.ref_order.argtypes = [C.c_int, _f64p, _i32p, _f64p]
        R.ref_pattern.restype = C.c_int64
        R.ref_pattern.argtypes = [C.c_int, _f64p, _i32p, _f64p, C.c_double, _i32p, C.c_void_p]
        _ref = R
    return _ref


def _pts(p):
    return np.ascontiguousarray(p, dtype=np.float64).reshape(-1, 3)


# --------------------------------------------------------------------------
# host-side plan: ordering, pattern, supernodes
# --------------------------------------------------------------------------

def order(pts):
    p = _pts(pts)
    n = p.shape[0]
    P = np.empty(n, np.int32)
    s = np.empty(n, np.float64)
    rc = lib().orc_order(n, p.ravel(), P, s)
    if rc:
        raise RuntimeError(f"oracle ordering failed ({rc})")
    return P, s


def ref_order(pts):
    p = _pts(pts)
    n = p.shape[0]
    P = np.empty(n, np.int32)
    s = np.empty(n, np.float64)
    rc = ref().ref_order(n, p.ravel(), P, s)
    if rc:
        raise RuntimeError(f"reference ordering failed ({rc})")
    return P, s


def pattern(pts, P, scale, rho):
    """MRA pattern in the new order; rho is widened from float32 like the reference."""
    p = _pts(pts)
    n = p.shape[0]
    pinv = np.empty(n, np.int32)
    pinv[P] = np.arange(n, dtype=np.int32)
    pp = np.ascontiguousarray(p[pinv])
    r = float(np.float32(rho))
    ptr = np.empty(n + 1, np.int32)
    nnz = lib().orc_pattern(n, pp.ravel(), scale, r, ptr, None)
    ind = np.empty(max(nnz, 1), np.int32)
    lib().orc_pattern(n, pp.ravel(), scale, r, ptr, _vp(ind))
    return ptr, ind[:nnz]


def ref_pattern(pts, P, scale, rho):
    p = _pts(pts)
    n = p.shape[0]
    r = float(np.float32(rho))
    ptr = np.empty(n + 1, np.int32)
    nnz = ref().ref_pattern(n, p.ravel(), P, scale, r, ptr, None)
    ind = np.empty(max(nnz, 1), np.int32)
    ref().ref_pattern(n, p.ravel(), P, scale, r, ptr, _vp(ind))
    return ptr, ind[:nnz]


def aggregate(ptr, ind, scale, lam=1.5, max_super=2048):
    n = ptr.shape[0] - 1
    sup_ptr = np.empty(n + 1, np.int32)
    sup_ind = np.empty(n, np.int32)
    sup_parent = np.empty(n, np.int32)
    ns = np.zeros(1, np.int32)
    rc = lib().orc_aggregate(n, ptr, np.ascontiguousarray(ind, np.int32), scale, lam, max_super,
                             sup_ptr, sup_ind, sup_parent, ns)
    if rc:
        raise RuntimeError(f"aggregation failed to cover every point ({rc})")
    return sup_ptr[:ns[0] + 1].copy(), sup_ind, sup_parent


def super_sets(ptr, ind, n_super, sup_parent):
    n = ptr.shape[0] - 1
    set_ptr = np.empty(n_super + 1, np.int32)
    ind = np.ascontiguousarray(ind, np.int32)
    tot = lib().orc_super_sets(n, ptr, ind, n_super, sup_parent, set_ptr, None)
    set_ind = np.empty(max(tot, 1), np.int32)
    lib().orc_super_sets(n, ptr, ind, n_super, sup_parent, set_ptr, _vp(set_ind))
    return set_ptr, set_ind[:tot]


def super_pattern(sup_parent, set_ptr, set_ind):
    n = sup_parent.shape[0]
    lptr = np.empty(n + 1, np.int32)
    set_ind = np.ascontiguousarray(set_ind, np.int32)
    nnz = lib().orc_super_pattern(n, sup_parent, set_ptr, set_ind, lptr, None)
    lind = np.empty(max(nnz, 1), np.int32)
    lib().orc_super_pattern(n, sup_parent, set_ptr, set_ind, lptr, _vp(lind))
    return lptr, lind[:nnz]


def plan(pts, rho=3.0, lam=1.5, max_super=2048):
    """Ordering + pattern + supernodes + supernodal pattern, as a dict."""
    P, scale = order(pts)
    ptr, ind = pattern(pts, P, scale, rho)
    sup_ptr, sup_ind, sup_parent = aggregate(ptr, ind, scale, lam, max_super)
    ns = sup_ptr.shape[0] - 1
    set_ptr, set_ind = super_sets(ptr, ind, ns, sup_parent)
    lptr, lind = super_pattern(sup_parent, set_ptr, set_ind)
    n = P.shape[0]
    pinv = np.empty(n, np.int32)
    pinv[P] = np.arange(n, dtype=np.int32)
    sizes = np.diff(set_ptr).astype(np.int64)
    th_ptr = np.zeros(ns + 1, np.int64)
    th_ptr[1:] = np.cumsum(sizes * sizes)
    return dict(P=P, Pinv=pinv, scale=scale, ptr=ptr, ind=ind, sup_ptr=sup_ptr,
                sup_ind=sup_ind, sup_parent=sup_parent, set_ptr=set_ptr, set_ind=set_ind,
                lptr=lptr, lind=lind, th_ptr=th_ptr, n_super=ns)


# --------------------------------------------------------------------------
# numeric: operator, factor, PCG (FP64)
# --------------------------------------------------------------------------

class Op:
    """Operator K: dense row-major M (nf x n) or the Laplace point kernel."""

    def __init__(self, nf, n, M=None, x=None, nx=None, y=None, coef=1.0):
        self.nf, self.n, self.coef = int(nf), int(n), float(coef)
        c = lambda a: None if a is None else np.ascontiguousarray(a, np.float64)
        self.M, self.x, self.nx, self.y = c(M), c(x), c(nx), c(y)

    @classmethod
    def from_scene(cls, sc):
        return cls(sc.nf, sc.n, x=sc.x, nx=sc.nx, y=sc.y, coef=sc.coef)

    def args(self):
        return (self.nf, self.n, _vp(self.M), _vp(self.x), _vp(self.nx), _vp(self.y), self.coef)

    def K(self, v):
        v = np.ascontiguousarray(v, np.float64)
        R = 1 if v.ndim == 1 else v.shape[1]
        w = np.empty((self.nf, R))
        lib().orc_apply_K(*self.args(), R, v.reshape(-1), w.reshape(-1))
        return w[:, 0] if v.ndim == 1 else w

    def KT(self, w):
        w = np.ascontiguousarray(w, np.float64)
        R = 1 if w.ndim == 1 else w.shape[1]
        t = np.empty((self.n, R))
        lib().orc_apply_KT(*self.args(), R, w.reshape(-1), t.reshape(-1))
        return t[:, 0] if w.ndim == 1 else t


def factor(op: Op, pl: dict):
    """Theta (reversed, Cholesky-factored in place) and the KL factor values."""
    th = np.empty(int(pl["th_ptr"][-1]), np.float64)
    lval = np.empty(pl["lind"].shape[0], np.float64)
    bad = C.c_int32(0)
    lib().orc_factor(*op.args(), pl["Pinv"], pl["n_super"], pl["sup_ptr"], pl["sup_ind"],
                     pl["set_ptr"], np.ascontiguousarray(pl["set_ind"], np.int32), pl["th_ptr"],
                     th, pl["lptr"], np.ascontiguousarray(pl["lind"], np.int32), lval,
                     C.byref(bad))
    return th, lval, int(bad.value)


def precond(pl, lval, r):
    n = r.shape[0]
    tmp = np.empty(n)
    z = np.empty(n)
    lib().orc_precond(n, pl["lptr"], np.ascontiguousarray(pl["lind"], np.int32), lval,
                      np.ascontiguousarray(r, np.float64), tmp, z)
    return z


def pcg(op: Op, pl: dict, lval, f=None, b=None, maxits=1000, tol=1e-8, precond=True):
    """One PCG solve in the NEW order; returns (x_new_order, iters, relres).

    Forward (b is None): solves K_p^T K_p x = K_p^T f (kl_chol.cu:891-1088).
    Adjoint (b given, new order): solves K_p^T K_p x = b (kl_chol.cu:1090-1264).
    """
    x = np.empty(op.n)
    rr = C.c_double(0.0)
    fa = None if f is None else np.ascontiguousarray(f, np.float64)
    ba = None if b is None else np.ascontiguousarray(b, np.float64)
    it = lib().orc_pcg(*op.args(), pl["Pinv"], pl["lptr"],
                       np.ascontiguousarray(pl["lind"], np.int32), lval,
                       1 if b is not None else 0, _vp(fa), _vp(ba), 1 if precond else 0,
                       int(maxits), float(tol), x, C.byref(rr))
    return x, it, rr.value


def pcg_many(op: Op, pl: dict, lval, F, maxits=1000, tol=1e-8):
    """orc_pcg on every column of F (nf x R) with shared K / K^T passes:
    per column the same x, iterations and relres as pcg(f=F[:, c]).
    Returns (X new order n x R, iters int32[R], relres[R])."""
    F = np.ascontiguousarray(np.atleast_2d(np.asarray(F, np.float64).T).T)
    R = F.shape[1]
    X = np.empty((op.n, R))
    its = np.empty(R, np.int32)
    rel = np.empty(R)
    if lib().orc_pcg_many(*op.args(), pl["Pinv"], pl["lptr"], np.ascontiguousarray(pl["lind"], np.int32),
                          lval, R, F.reshape(-1), int(maxits), float(tol), X.reshape(-1), its, rel) != 0:
        raise MemoryError("orc_pcg_many")
    return X, its, rel


def solve(op: Op, pl: dict, lval, F, maxits=1000, tol=1e-8):
    """All columns of F (nf x R); returns strengths in ORIGINAL order (n x R)."""
    F = np.atleast_2d(np.asarray(F, np.float64).T).T
    X = np.empty((op.n, F.shape[1]))
    its = []
    for r in range(F.shape[1]):
        xn, it, _ = pcg(op, pl, lval, f=F[:, r], maxits=maxits, tol=tol)
        X[:, r] = xn[pl["P"]]
        its.append(it)
    return X, its


def added_mass(sc, X, rho_f=1.0):
    """Added-mass tensor (6 bodies x R) of strengths X (n x R, original order)
    for a scene with area weights; FP64 (orc_added_mass)."""
    X = np.ascontiguousarray(np.atleast_2d(np.asarray(X, np.float64).T).T)
    R = X.shape[1]
    nb = sc.n_bodies
    out = np.empty((6 * nb, R))
    f = lambda a: np.ascontiguousarray(a, np.float64)
    lib().orc_added_mass(sc.nf, sc.n, f(sc.x), f(sc.nx), f(sc.y), R, X, f(sc.weights()), nb,
                         np.ascontiguousarray(sc.body_ptr(), np.int32), f(sc.centers), float(rho_f), out)
    return out


def mesh_operator(V, F, face_body, body_pos, S):
    """Solid-angle matrix (faces x sources) and rigid-mode right-hand side
    FL @ IQ (faces x 6 bodies) of a triangle-mesh scene, FP64."""
    f = lambda a: np.ascontiguousarray(a, np.float64)
    i = lambda a: np.ascontiguousarray(a, np.int32)
    V, F, S, fb, bp = f(V), i(F), f(S), i(face_body), f(body_pos)
    nfc, ns, nb = F.shape[0], S.shape[0], bp.shape[0]
    M = np.empty((nfc, ns))
    rhs = np.empty((nfc, 6 * nb))
    lib().orc_mesh_solid_angle(nfc, V, F, ns, S, M)
    lib().orc_mesh_rhs(nfc, V, F, fb, nb, bp, rhs)
    return M, rhs


def oz_apply(G, V, coef=1.0):
    """coef * G @ V through the INT8 digit-sliced FP64 matvec, computed the
    way the library's INT8 tensor-core kernels compute it (orc_oz_apply).
    Raises if a digit-level sum would overflow INT32."""
    G = np.ascontiguousarray(G, np.float64)
    V = np.asarray(V, np.float64)
    one = V.ndim == 1
    V = np.ascontiguousarray(V[:, None] if one else V)
    M, K = G.shape
    R = V.shape[1]
    assert V.shape[0] == K
    out = np.empty((M, R))
    if lib().orc_oz_apply(M, K, R, G, V, float(coef), out) != 0:
        raise OverflowError("INT8 digit-level sum outside the INT32 range")
    return out[:, 0] if one else out


def num_threads() -> int:
    return int(lib().orc_num_threads())
