"""The FP64-accurate INT8 tensor-core matvec (mbc_solver_set_fp64_matvec) on
the GPU, against the oracle's restatement of the same integer pipeline
(orc_oz_apply) and against the FP64 CUDA-core kernels.

Tolerances (per element, with bound(G, V) = 2^-33 sum_c kc max|G_c| max|V_c|,
the scheme's worst-case error; kc = 2048-wide chunk length):
  * device vs oracle: <= bound / 64 (the two evaluate G in FP64 by different
    rsqrt routes, so a digit can differ by one unit where G lies within an
    ulp of a rounding tie);
  * device vs FP64 kernels: <= bound, and 1e-9 relative norm-wise;
  * solves: FP64 true relative residual <= 1.05e-8 per column (the FP64
    kernels recompute it), at most 25 % + one check block more iterations
    than the FP64 kernels (the operator's ~1e-9 relative product error slows
    the ill-conditioned columns: 264 against 225 on this scene, measured on
    the B200), fitted flux within 1e-6 of theirs (relative to |F|).
"""
import numpy as np
import pytest

import fastmbcui_b200 as F
import oracle as O
from fastmbcui_b200 import _lib
from fastmbcui_b200 import scenes as S

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
CHUNK = 2048


def _dev(a, dt=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")


def _G(sc):
    """The point kernel without coef, FP64 from the float32-exact coordinates."""
    r = sc.x[:, None, :] - sc.y[None, :, :]
    r2 = (r[..., 0] * r[..., 0] + r[..., 1] * r[..., 1]) + r[..., 2] * r[..., 2]
    rn = (r[..., 0] * sc.nx[:, None, 0] + r[..., 1] * sc.nx[:, None, 1]) + r[..., 2] * sc.nx[:, None, 2]
    return rn / (np.sqrt(r2) * r2)


def _bound(G, V, coef):
    b = np.zeros((G.shape[0], V.shape[1]))
    for k0 in range(0, G.shape[1], CHUNK):
        kc = min(CHUNK, G.shape[1] - k0)
        b += np.abs(G[:, k0:k0 + kc]).max(axis=1)[:, None] * np.abs(V[k0:k0 + kc]).max(axis=0)[None, :] * kc
    return abs(coef) * 2.0 ** -33 * b


class Case:
    def __init__(self):
        # n = nf = 3000: two 2048-wide chunks, a ragged last k-step and row tile
        self.sc = sc = S.ellipsoids_scene(2, 1500, seed=11)
        self.plan = F.Plan(sc.y, sc.rho, sc.lam, sc.max_super)
        x, nx, y = _dev(sc.x, torch.float32), _dev(sc.nx, torch.float32), _dev(sc.y, torch.float32)
        self.s64 = F.Solver(self.plan, x=x, nx=nx, y=y, coef=sc.coef, precision=F.MBC_F64)
        self.s8 = F.Solver(self.plan, x=x, nx=nx, y=y, coef=sc.coef, precision=F.MBC_F64).set_fp64_matvec("int8")
        self.s32 = F.Solver(self.plan, x=x, nx=nx, y=y, coef=sc.coef, precision=F.MBC_F32).set_fp64_matvec("int8")
        P, _ = self.plan.order()
        self.P = P.astype(np.int64)
        self.Pinv = np.argsort(self.P)
        self.G = _G(sc)
        # the planes' reduction axes walk the sources (K) and the rows (K^T)
        # in Morton order; the sources are given to it in plan order
        self.ks = self.Pinv[F.spatial_order(sc.y[self.Pinv])]  # original source indices along K's axis
        self.kr = F.spatial_order(sc.x).astype(np.int64)      # row indices along K^T's axis


@pytest.fixture(scope="module")
def case():
    return Case()


@pytest.mark.parametrize("R", [1, 12, 100, 192])
def test_apply_K(case, R):
    sc = case.sc
    V = np.random.default_rng(R).standard_normal((sc.n, R))
    W8 = case.s8.apply_K(_dev(V)).cpu().numpy().reshape(sc.nf, R)
    W64 = case.s64.apply_K(_dev(V)).cpu().numpy().reshape(sc.nf, R)
    Gn, Vn = case.G[:, case.ks], V[case.ks]  # the device's reduction order
    Wo = O.oz_apply(Gn, Vn, coef=sc.coef)
    bound = _bound(Gn, Vn, sc.coef)
    assert np.all(np.abs(W8 - Wo) <= bound / 64)
    assert np.all(np.abs(W8 - W64) <= bound)
    assert np.linalg.norm(W8 - W64) / np.linalg.norm(W64) <= 1e-9


@pytest.mark.parametrize("R", [1, 12, 192])
def test_apply_KT(case, R):
    sc = case.sc
    W = np.random.default_rng(100 + R).standard_normal((sc.nf, R))
    T8 = case.s8.apply_KT(_dev(W)).cpu().numpy().reshape(sc.n, R)
    T64 = case.s64.apply_KT(_dev(W)).cpu().numpy().reshape(sc.n, R)
    GnT = np.ascontiguousarray(case.G[case.kr][:, case.Pinv].T)  # sources (plan order) x rows (Morton)
    Wk = W[case.kr]
    To = O.oz_apply(GnT, Wk, coef=sc.coef)[case.P]               # back to the original order
    bound = _bound(GnT, Wk, sc.coef)[case.P]
    assert np.all(np.abs(T8 - To) <= bound / 64)
    assert np.all(np.abs(T8 - T64) <= bound)
    assert np.linalg.norm(T8 - T64) / np.linalg.norm(T64) <= 1e-9


def test_fp64_solve_on_int8_matvec(case):
    sc = case.sc
    op = O.Op.from_scene(sc)
    Fm = sc.rhs()
    case.s64.factor()
    case.s8.factor()
    X64, st64 = case.s64.solve(_dev(Fm), tol=1e-8, max_iters=4000)
    X8, st8 = case.s8.solve(_dev(Fm), tol=1e-8, max_iters=4000, true_residual=1)
    X8, X64 = X8.cpu().numpy(), X64.cpu().numpy()
    b = op.KT(Fm)
    rel = np.linalg.norm(op.KT(Fm - op.K(X8)), axis=0) / np.linalg.norm(b, axis=0)
    assert rel.max() <= 1.05e-8, rel
    assert st8["true_relres_max"] <= 1.05e-8
    assert st8["iters_max"] <= 1.25 * st64["iters_max"] + 8, (st8["iters_max"], st64["iters_max"])
    assert np.linalg.norm(op.K(X8) - op.K(X64)) / np.linalg.norm(Fm) < 1e-6


def test_mixed_solve_polishes_on_int8_matvec(case):
    sc = case.sc
    op = O.Op.from_scene(sc)
    Fm = sc.rhs()
    case.s32.factor()
    X, st = case.s32.solve(_dev(Fm, torch.float32), out_dtype=torch.float64, tol=1e-8, max_iters=4000)
    X = X.cpu().numpy()
    b = op.KT(Fm)
    rel = np.linalg.norm(op.KT(Fm - op.K(X)), axis=0) / np.linalg.norm(b, axis=0)
    assert rel.max() <= 1.05e-8, (rel, st)


def test_int8_needs_a_point_kernel():
    sc = S.ellipsoids_scene(1, 300, seed=2)
    plan = F.Plan(sc.y, sc.rho, sc.lam, sc.max_super)
    M = _dev(sc.dense_K(), torch.float32)
    s = F.Solver(plan, M=M, precision=F.MBC_F64)
    with pytest.raises(F.MbcError):
        s.set_fp64_matvec("int8")
    with pytest.raises(F.MbcError):
        s.set_fp64_matvec(7)
    assert _lib.MBC_FP64_MATVEC_INT8 == F.MBC_FP64_MATVEC_INT8
