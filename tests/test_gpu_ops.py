"""The drop-in mfs_torch operators on the GPU, against the FP64 oracle.

The operators compute in FP32 (vectors, matvec, factor) with FP64 PCG
scalars, like the reference's FP32 path; tolerances are stated per check.
"""
import numpy as np
import pytest

import oracle as O
from fastmbcui_b200 import scenes as S

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def setup():
    import fastmbcui_b200.mfs_torch as mfs

    sc = S.ellipsoids_scene(2, 1200, seed=8)
    K = sc.dense_K().astype(np.float32)
    op = O.Op(sc.nf, sc.n, M=K.astype(np.float64))
    pl = O.plan(sc.y, 3.0)
    _, lval, _ = O.factor(op, pl)
    return mfs, sc, K, op, pl, lval


def _t(a, dt=torch.float32, dev="cuda"):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)


def test_minvf_matches_oracle(setup):
    mfs, sc, K, op, pl, lval = setup
    Fm = sc.rhs()
    out = mfs.ops.MinvF_float_fastGrad(_t(K), _t(Fm), _t(sc.y, dev="cpu"), 3.0, 1000, 1e-5)
    X = out.double().cpu().numpy()
    assert out.shape == (sc.n, Fm.shape[1]) and out.dtype == torch.float32
    for c in range(Fm.shape[1]):
        xo, it, rr = O.pcg(op, pl, lval, f=Fm[:, c], maxits=1000, tol=1e-5)
        # fitted boundary flux agrees to FP32-PCG accuracy (relative to |f|)
        d = np.linalg.norm(op.K(X[:, c]) - op.K(xo[pl["P"]])) / np.linalg.norm(Fm[:, c])
        assert d < 1e-3, (c, d)


def test_minvf_reference_demo_settings(setup):
    # rho 1.2, 75 iterations, tol 2.7e-3 (simuspclf1d_mfs_coins.py:21-23)
    mfs, sc, K, op, _, _ = setup
    pl = O.plan(sc.y, 1.2)
    _, lval, _ = O.factor(op, pl)
    Fm = sc.rhs()[:, :4]
    out = mfs.ops.MinvF_float_fastGrad(_t(K), _t(Fm), _t(sc.y, dev="cpu"), 1.2, 75, 2.7e-3)
    X = out.double().cpu().numpy()
    for c in range(4):
        xo, it, rr = O.pcg(op, pl, lval, f=Fm[:, c], maxits=75, tol=2.7e-3)
        d = np.linalg.norm(op.K(X[:, c]) - op.K(xo[pl["P"]])) / np.linalg.norm(Fm[:, c])
        assert d < 2e-2, (c, d)


def test_vpl_matches_oracle_adjoint(setup):
    mfs, sc, K, op, pl, lval = setup
    Fm = sc.rhs()[:, :3]
    Vs = _t(sc.y, dev="cpu")
    mfs.ops.MinvF_float_fastGrad(_t(K), _t(Fm), Vs, 3.0, 1000, 1e-6)
    rng = np.random.default_rng(0)
    G = rng.standard_normal((sc.n, 3)).astype(np.float32)
    V = mfs.ops.VpL_fast_float(_t(K), _t(G), Vs, 3.0, 2000, 1e-6).double().cpu().numpy()
    for c in range(3):
        xo, it, rr = O.pcg(op, pl, lval, b=G[pl["Pinv"], c].astype(np.float64), maxits=4000, tol=1e-10)
        # K v is what the autograd formula consumes (grad_F = M VpL); the
        # FP32-rounded v itself is ill-conditioned
        kv, kvo = op.K(V[:, c]), op.K(xo[pl["P"]])
        assert np.linalg.norm(kv - kvo) / np.linalg.norm(kvo) < 1e-3


def test_autograd_formula(setup):
    mfs, sc, K, op, pl, lval = setup
    Fm = sc.rhs()[:, :2]
    M = _t(K).requires_grad_(True)
    Ft = _t(Fm).requires_grad_(True)
    Vs = _t(sc.y, dev="cpu")
    A = mfs.ops.MinvF_float_fastGrad(M, Ft, Vs, 3.0, 2000, 1e-7)
    rng = np.random.default_rng(3)
    G = _t(rng.standard_normal((sc.n, 2)))
    (A * G).sum().backward()
    # dense FP64: grad_F = M (M^T M)^{-1} G
    K64 = K.astype(np.float64)
    N = K64.T @ K64
    VpL = np.linalg.solve(N, G.double().cpu().numpy())
    gF = K64 @ VpL
    assert np.linalg.norm(Ft.grad.double().cpu().numpy() - gF) / np.linalg.norm(gF) < 2e-2
    # grad_M = -M (W + W^T) + F VpL^T with W = A VpL^T
    A64 = A.detach().double().cpu().numpy()
    W = A64 @ VpL.T
    gM = -K64 @ (W + W.T) + Fm @ VpL.T
    assert np.linalg.norm(M.grad.double().cpu().numpy() - gM) / np.linalg.norm(gM) < 2e-2


def test_vpl_before_forward_is_refused():
    import ctypes as C

    import fastmbcui_b200 as F

    L = F.load()
    h = C.c_void_p()
    assert L.mbc_context_create(C.byref(h)) == 0
    x = torch.zeros((4, 4), device="cuda")
    pts = np.zeros((4, 3), np.float32)
    s = L.mbc_vpl_fast_float(h, x.data_ptr(), 4, 4, x.data_ptr(), 1, pts.ctypes.data, 3.0, 10, 1e-3, 0, 0,
                             x.data_ptr(), None)
    assert s == 4 and b"MinvF_float first" in L.mbc_last_error()
    L.mbc_context_destroy(h)


def test_argument_checks(setup):
    mfs, sc, K, op, pl, lval = setup
    M, Fm, Vs = _t(K), _t(sc.rhs()), _t(sc.y, dev="cpu")
    with pytest.raises(RuntimeError, match="F must be a 2D tensor"):
        mfs.ops.MinvF_float_fastGrad(M, Fm[:, 0], Vs, 3.0, 10, 1e-3)
    with pytest.raises(RuntimeError, match="same first dimension"):
        mfs.ops.MinvF_float_fastGrad(M[:-1], Fm, Vs, 3.0, 10, 1e-3)
    with pytest.raises(RuntimeError, match="compatible dimensions"):
        mfs.ops.MinvF_float_fastGrad(M, Fm, Vs[:-1], 3.0, 10, 1e-3)
    with pytest.raises(RuntimeError):
        mfs.ops.MinvF_float_fastGrad(M, Fm, Vs.cuda(), 3.0, 10, 1e-3)
    with pytest.raises(RuntimeError):
        mfs.ops.MinvF_float_fastGrad(M.double(), Fm, Vs, 3.0, 10, 1e-3)
    with pytest.raises(NotImplementedError):
        mfs.ops.MinvF_float_fastGrad(M.cpu(), Fm.cpu(), Vs, 3.0, 10, 1e-3)


def test_lowrank_gradient_kernel_matches_dense_formula():
    """mbc_minvf_grad against the reference's dense backward formula
    (core/mfs_torch_py/ops.py:52-57) evaluated in FP64: grad_M and grad_F
    within 1e-5 relative (FP32 products of 500 and 14 terms)."""
    import ctypes as C

    from fastmbcui_b200 import _lib

    g = torch.Generator(device="cuda").manual_seed(3)
    nf, n, R = 700, 500, 7
    M = torch.randn(nf, n, generator=g, device="cuda")
    F = torch.randn(nf, R, generator=g, device="cuda")
    A = torch.randn(n, R, generator=g, device="cuda")
    V = torch.randn(n, R, generator=g, device="cuda")
    work = torch.empty(nf, 2 * R, device="cuda")
    gM, gF = torch.empty_like(M), torch.empty_like(F)
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(_lib.load().mbc_minvf_grad(nf, n, R, M.data_ptr(), n, F.data_ptr(), A.data_ptr(), V.data_ptr(),
                                          work.data_ptr(), gM.data_ptr(), n, gF.data_ptr(), st), "mbc_minvf_grad")
    Md, Fd, Ad, Vd = (t.double() for t in (M, F, A, V))
    W = Ad @ Vd.T
    want_M = -Md @ (W + W.T) + Fd @ Vd.T
    want_F = Md @ Vd
    assert float(torch.linalg.norm(gM.double() - want_M) / torch.linalg.norm(want_M)) < 1e-5
    assert float(torch.linalg.norm(gF.double() - want_F) / torch.linalg.norm(want_F)) < 1e-5
