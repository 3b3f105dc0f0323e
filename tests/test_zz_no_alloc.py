"""mbc_point_apply_noalloc: the point-kernel matvec with a static workspace.

Its output is checked against the FP64 oracle's K / K^T (oracle.Op, the CPU
restatement of the point kernel) and against the library's allocating entry
points (the solver's mbc_apply_K / mbc_apply_KT) on the same points, within
the FP32 matvec tolerance of the other parity tests (2e-5, norm-wise
relative), over calls in a row that reuse the shared static array with
different sizes and directions.
"""
import ctypes as C

import numpy as np
import pytest

import fastmbcui_b200 as F
import oracle as O
from fastmbcui_b200 import _lib
from fastmbcui_b200 import scenes as S

torch = pytest.importorskip("torch")

TOL = 2e-5


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _dev(a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float32, device="cuda")


def noalloc(transpose, x, nx, y, coef, V):
    nf, n, R = x.shape[0], y.shape[0], V.shape[1]
    out = torch.empty((n if transpose else nf, R), dtype=torch.float32, device="cuda")
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(F.load().mbc_point_apply_noalloc(transpose, nf, n, x.data_ptr(), nx.data_ptr(), y.data_ptr(),
                                                 coef, R, V.data_ptr(), out.data_ptr(), st),
               "mbc_point_apply_noalloc")
    return out


class Scene:
    def __init__(self, sc):
        self.sc = sc
        self.x, self.nx, self.y = _dev(sc.x), _dev(sc.nx), _dev(sc.y)
        plan = F.Plan(sc.y, sc.rho, sc.lam, sc.max_super)
        self.solver = F.Solver(plan, x=self.x, nx=self.nx, y=self.y, coef=sc.coef, precision=F.MBC_F32)
        self.op = O.Op.from_scene(sc)

    def check(self, transpose, R, seed):
        rng = np.random.default_rng(seed)
        Vh = rng.standard_normal((self.sc.nf if transpose else self.sc.n, R)).astype(np.float32)
        V = _dev(Vh)
        got = noalloc(transpose, self.x, self.nx, self.y, self.sc.coef, V)
        lib = self.solver.apply_KT(V) if transpose else self.solver.apply_K(V)
        torch.cuda.synchronize()
        got = got.double().cpu().numpy()
        oracle = self.op.KT(Vh) if transpose else self.op.K(Vh)
        err = rel(got, oracle)
        assert err < TOL, (transpose, R, err)
        assert rel(got, lib.double().cpu().numpy()) < TOL, (transpose, R)


@pytest.mark.gpu
def test_noalloc_matches_solver_matvec_on_calls_in_a_row():
    big = Scene(S.ellipsoids_scene(3, 1500, seed=21))
    small = Scene(S.ellipsoids_scene(2, [333, 517], seed=22))
    # the second call reads the array where the first left larger contents
    big.check(0, 24, 1)
    small.check(1, 5, 2)
    small.check(0, 1, 3)
    big.check(1, 40, 4)


@pytest.mark.gpu
def test_noalloc_largest_accepted_size():
    # 2*nf + n at the static limit: 87376 rows and 87376 sources use 262128 slots
    rng = np.random.default_rng(5)
    n = 87376
    y = rng.standard_normal((n, 3)).astype(np.float32)
    y /= np.linalg.norm(y, axis=1, keepdims=True)
    x, nx, y = 1.5 * y, y.copy(), 0.8 * y
    coef = S.COEF_LAPLACE_DN
    xd, nxd, yd = _dev(x), _dev(nx), _dev(y)
    V = _dev(rng.standard_normal((n, 2)))
    got = noalloc(0, xd, nxd, yd, coef, V).double().cpu().numpy()
    # FP64 check on a few rows
    rows = rng.choice(n, 16, replace=False)
    d = x[rows, None, :].astype(np.float64) - y[None, :, :].astype(np.float64)
    r2 = (d * d).sum(-1)
    k = (d * nx[rows, None, :].astype(np.float64)).sum(-1) / (r2 * np.sqrt(r2))
    want = coef * k @ V.double().cpu().numpy()
    assert rel(got[rows], want) < TOL


def test_noalloc_refuses_overlapping_buffers():
    L = F.load()
    p = C.c_void_p(4096)
    # out starts inside in's 10 x 2 floats (80 bytes): refused before any launch
    s = L.mbc_point_apply_noalloc(0, 10, 10, p, p, p, 1.0, 2, C.c_void_p(4096), C.c_void_p(4096 + 40), None)
    assert s == _lib.MBC_BAD_ARG
    assert b"overlap" in L.mbc_last_error()
    s = L.mbc_point_apply_noalloc(1, 10, 10, p, p, p, 1.0, 2, C.c_void_p(4096), C.c_void_p(4096), None)
    assert s == _lib.MBC_BAD_ARG


def test_noalloc_refuses_sizes_beyond_the_static_scratch():
    L = F.load()
    p = C.c_void_p(16)
    s = L.mbc_point_apply_noalloc(0, 100000, 70000, p, p, p, 1.0, 1, p, p, None)
    assert s == _lib.MBC_BAD_ARG
    assert b"exceed the static scratch" in L.mbc_last_error()
    assert L.mbc_point_apply_noalloc(2, 10, 10, p, p, p, 1.0, 1, p, p, None) == _lib.MBC_BAD_ARG
    assert L.mbc_point_apply_noalloc(0, 0, 10, p, p, p, 1.0, 1, p, p, None) == _lib.MBC_BAD_ARG
