"""The learned warm start on a small trajectory, against the method without it
(the previous step's strengths).

Over held-out steps the trained network must predict its targets (relative
error below 0.5) and start the PCG at a lower FP64-recomputed normal-equation
residual |K^T (f - K x0)| / |K^T f| than the previous step's strengths.  The
FP64 PCG iterations to 1e-8 from both starts (stopping tested every
iteration) are measured and reported: a lower starting residual does not by
itself save iterations -- measured here, the correction in the isolated-body
basis costs iterations, because it adds error along the operator's
ill-conditioned directions -- so the trajectory benchmark starts from the
previous step.
"""
import numpy as np
import pytest

import fastmbcui_b200 as F
import oracle as O
from fastmbcui_b200 import scenes as S
from fastmbcui_b200 import warmstart as W
from fastmbcui_b200.train_warmstart import generate, train

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _t(a):
    return torch.as_tensor(np.ascontiguousarray(a, np.float32), device="cuda")


def test_warm_correct_kernel():
    sc = S.ellipsoids_scene(3, [20, 30, 25], seed=1)
    rng = np.random.default_rng(0)
    U = rng.standard_normal((sc.n, 6)).astype(np.float32)
    H = rng.standard_normal((3 * 3, 36)).astype(np.float32)
    X = rng.standard_normal((sc.n, 18)).astype(np.float32)
    want = X.astype(np.float64).copy()
    for j in range(sc.n):
        c = sc.src_body[j]
        for b in range(3):
            want[j, 6 * b:6 * b + 6] += U[j].astype(np.float64) @ H[c * 3 + b].reshape(6, 6)
    ws = W.WarmStart(None, 0, 1, 1.0)
    Xd = _t(X)
    import ctypes as C
    from fastmbcui_b200 import _lib
    sb = torch.as_tensor(sc.src_body, dtype=torch.int32, device="cuda")
    Ud, Hd = _t(U), _t(H)
    _lib.check(F.load().mbc_warm_correct(sc.n, 18, sb.data_ptr(), 3, Ud.data_ptr(), Hd.data_ptr(), Xd.data_ptr(),
                                         C.c_void_p(torch.cuda.current_stream().cuda_stream)), "warm")
    got = Xd.double().cpu().numpy()
    assert np.abs(got - want).max() < 1e-5 * np.abs(want).max()
    del ws


def test_learned_warm_start_gains_over_previous_step():
    steps, pts, nb, seed = 24, 400, 6, 7
    feats, targs, iters = generate(pts, steps, seed, n_bodies=nb)
    ws, info = train(feats, targs, epochs=300, hold=0.25)
    assert info["val_rel_err"] < 0.5, info
    # replay the held-out steps: starting residual of x(t-1) vs x(t-1) + U H
    base, q, _ = S.trajectory_scene(nb, pts, seed=seed, steps=steps + 1)
    U = W.isolated_basis(base)
    sb = torch.as_tensor(base.src_body, dtype=torch.int32, device="cuda")
    X_prev = None
    r_prev, r_learn, it_prev, it_learn = [], [], [], []
    first_eval = int(round(steps * 0.75)) + 1
    for k in range(steps + 1):
        sc = S.moved(base, q[k])
        plan = F.Plan(sc.y, sc.rho, sc.lam, sc.max_super)
        s = F.Solver(plan, x=_t(sc.x), nx=_t(sc.nx), y=_t(sc.y), coef=sc.coef, precision=F.MBC_F32).factor()
        Fm = sc.rhs()
        opts = dict(out_dtype=torch.float32, tol=1e-8, max_iters=4000, max_refine=64, inner_tol=1e-2)
        if X_prev is not None and k >= first_eval:
            pairs = W.neighbour_pairs(sc.centers)
            f = W.pair_features(pairs, q[k - 1], q[k], base.centers, base.meta["axes"], base.meta["rot"])
            X0 = ws.apply(X_prev, U, sb, nb, pairs, f)
            op = O.Op.from_scene(sc)
            b = op.KT(Fm)
            rel = lambda X: np.linalg.norm(op.KT(Fm - op.K(X))) / np.linalg.norm(b)
            r_prev.append(rel(X_prev.double().cpu().numpy()))
            r_learn.append(rel(X0.double().cpu().numpy()))
            s64 = F.Solver(plan, x=_t(sc.x), nx=_t(sc.nx), y=_t(sc.y), coef=sc.coef,
                           precision=F.MBC_F64).factor()
            o64 = dict(tol=1e-8, max_iters=4000, check_every=1)
            _, st1 = s64.solve(_t(Fm).double(), X0=X_prev.double(), **o64)
            _, st2 = s64.solve(_t(Fm).double(), X0=X0.double(), **o64)
            it_prev.append(st1["iters_total"])
            it_learn.append(st2["iters_total"])
        X, _ = s.solve(_t(Fm), X0=X_prev, **opts)
        X_prev = X
    assert len(r_prev) >= 4
    assert np.mean(r_learn) < 0.7 * np.mean(r_prev), (r_learn, r_prev)
    print(f"\nstarting residual  previous {np.mean(r_prev):.3e}  learned {np.mean(r_learn):.3e}")
    print(f"FP64 PCG iterations (sum over columns)  previous {it_prev}  learned {it_learn}")


def test_cold_start_from_isolated_bodies():
    """A pose with no history (the plain method starts from x0 = 0).

    * x0 = each body's isolated rigid-mode solution at its pose (no network):
      must take fewer FP64 PCG iterations than x0 = 0 (measured ~27 % fewer);
    * plus the network's neighbour blocks (self blocks kept exact): measured
      and reported beside them.
    FP64 PCG to 1e-8, stopping tested every iteration, held-out poses."""
    from fastmbcui_b200.train_warmstart import generate_cold

    steps, pts, nb, seed = 24, 400, 6, 11
    feats, targs = generate_cold(pts, steps, seed, n_bodies=nb, stride=2)
    ws, info = train(feats, targs, epochs=300, hold=0.25, cls=W.ColdStart)
    base, q, _ = S.trajectory_scene(nb, pts, seed=seed, steps=steps * 2 + 1)
    U = W.isolated_basis(base)
    sb = torch.as_tensor(base.src_body, dtype=torch.int32, device="cuda")
    it_zero, it_iso, it_learn = [], [], []
    for k in range(int(round(steps * 0.75)) * 2, steps * 2, 2):
        sc = S.moved(base, q[k])
        plan = F.Plan(sc.y, sc.rho, sc.lam, sc.max_super)
        s64 = F.Solver(plan, x=_t(sc.x), nx=_t(sc.nx), y=_t(sc.y), coef=sc.coef, precision=F.MBC_F64).factor()
        Fm = _t(sc.rhs()).double()
        o64 = dict(tol=1e-8, max_iters=4000, check_every=1)
        R = Fm.shape[1]
        pairs = W.neighbour_pairs(sc.centers)
        f = W.cold_features(pairs, q[k], base.centers, base.meta["axes"], base.meta["rot"])
        x_iso = W.isolated_start(sc.n, R, U, sb, nb, q[k])
        x_learn = ws.start(sc.n, R, U, sb, nb, pairs, f, q[k])
        it_zero.append(s64.solve(Fm, **o64)[1]["iters_total"])
        it_iso.append(s64.solve(Fm, X0=x_iso.double(), **o64)[1]["iters_total"])
        it_learn.append(s64.solve(Fm, X0=x_learn.double(), **o64)[1]["iters_total"])
    print(f"\ncold-start FP64 iterations  zero {it_zero}  isolated {it_iso}  isolated + network {it_learn}"
          f"  (val rel err {info['val_rel_err']:.3f})")
    assert sum(it_iso) < 0.9 * sum(it_zero), (it_iso, it_zero)
