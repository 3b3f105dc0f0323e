"""Train the warm-start network on solves the method generates along a trajectory.

    python -m fastmbcui_b200.train_warmstart [--pts 500] [--steps 48] [--seed 100]
        [--out fastmbcui_b200/data/warmstart_mlp.npz]

A seeded 32-ellipsoid trajectory (``--pts`` points per body) is solved step
by step with the mixed-precision solver (each step warm-started from the
previous one); for every body b and each of its neighbours c the target is the
6 x 6 block that carries the previous strengths of body c for the modes of b
to the new ones in the isolated-body basis.  The MLP (3 x 256 tanh, BF16
weights, FP32 accumulation) is trained with the library's own kernels; the
last quarter of the steps is held out.  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np


def generate(pts, steps, seed, tol=1e-8, n_bodies=32):
    import torch

    from . import Plan, Solver, _lib
    from . import scenes as S
    from . import warmstart as W

    base, q, _ = S.trajectory_scene(n_bodies, pts, seed=seed, steps=steps + 1)
    U = W.isolated_basis(base)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32), device="cuda")
    X_prev, feats, targs, iters = None, [], [], []
    for k in range(steps + 1):
        sc = S.moved(base, q[k])
        plan = Plan(sc.y, sc.rho, sc.lam, sc.max_super)
        s = Solver(plan, x=t(sc.x), nx=t(sc.nx), y=t(sc.y), coef=sc.coef, precision=_lib.MBC_F32).factor()
        X, st = s.solve(t(sc.rhs()), X0=X_prev, out_dtype=torch.float32, tol=tol, max_iters=4000,
                        max_refine=64, inner_tol=1e-2)
        iters.append(int(st["iters_max"]))
        if X_prev is not None:
            pairs = W.neighbour_pairs(sc.centers)
            feats.append(W.pair_features(pairs, q[k - 1], q[k], base.centers, base.meta["axes"], base.meta["rot"]))
            targs.append(W.pair_targets(U, X - X_prev, base, pairs).cpu().numpy())
        X_prev = X
    return np.stack(feats), np.stack(targs), iters


def generate_cold(pts, steps, seed, tol=1e-8, n_bodies=32, stride=1):
    """Cold-start samples: for the poses of a trajectory, the pair features of
    each pose and the blocks H with U H = the solved strengths."""
    import torch

    from . import Plan, Solver, _lib
    from . import scenes as S
    from . import warmstart as W

    base, q, _ = S.trajectory_scene(n_bodies, pts, seed=seed, steps=steps * stride + 1)
    U = W.isolated_basis(base)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32), device="cuda")
    X_prev, feats, targs = None, [], []
    for k in range(0, steps * stride, stride):
        sc = S.moved(base, q[k])
        plan = Plan(sc.y, sc.rho, sc.lam, sc.max_super)
        s = Solver(plan, x=t(sc.x), nx=t(sc.nx), y=t(sc.y), coef=sc.coef, precision=_lib.MBC_F32).factor()
        X, _ = s.solve(t(sc.rhs()), X0=X_prev, out_dtype=torch.float32, tol=tol, max_iters=4000,
                       max_refine=64, inner_tol=1e-2)
        pairs = W.neighbour_pairs(sc.centers)
        feats.append(W.cold_features(pairs, q[k], base.centers, base.meta["axes"], base.meta["rot"]))
        targs.append(W.pair_targets(U, X, base, pairs).cpu().numpy())
        X_prev = X
    return np.stack(feats), np.stack(targs)


def train(feats, targs, epochs=400, batch=1024, lr=1e-3, seed=0, hold=0.25, cls=None):
    import torch

    from .warmstart import Mlp, WarmStart

    cls = cls or WarmStart

    T = feats.shape[0]
    n_tr = max(1, int(round(T * (1 - hold))))
    Xtr, Ytr = feats[:n_tr].reshape(-1, feats.shape[-1]), targs[:n_tr].reshape(-1, targs.shape[-1])
    Xva, Yva = feats[n_tr:].reshape(-1, feats.shape[-1]), targs[n_tr:].reshape(-1, targs.shape[-1])
    x_mean, x_std = Xtr.mean(0), Xtr.std(0) + 1e-6
    y_std = float(Ytr.std()) + 1e-30
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32), device="cuda")
    xs = dev((Xtr - x_mean) / x_std)
    ys = dev(Ytr / y_std)
    net = Mlp(Xtr.shape[1], Ytr.shape[1], hidden=256, layers=3, seed=seed)
    rng = np.random.default_rng(seed)
    hist = []
    for ep in range(epochs):
        perm = torch.as_tensor(rng.permutation(xs.shape[0]), device="cuda")
        for i in range(0, xs.shape[0], batch):
            idx = perm[i:i + batch]
            loss = net.train_step(xs[idx], ys[idx], lr=lr)
        if ep % 50 == 0 or ep == epochs - 1:
            hist.append((ep, loss))
    ws = cls(net, x_mean, x_std, y_std)

    def rel_err(X, Y):
        if X.shape[0] == 0:
            return None
        P = ws.predict_H(X).cpu().numpy()
        return float(np.linalg.norm(P - Y) / np.linalg.norm(Y))

    return ws, {"train_rel_err": rel_err(Xtr, Ytr), "val_rel_err": rel_err(Xva, Yva), "loss": hist,
                "samples_train": int(Xtr.shape[0]), "samples_val": int(Xva.shape[0])}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pts", type=int, default=500)
    ap.add_argument("--steps", type=int, default=48)
    ap.add_argument("--seed", type=int, default=100)
    ap.add_argument("--epochs", type=int, default=400)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(__file__), "data", "warmstart_mlp.npz"))
    a = ap.parse_args()
    t0 = time.perf_counter()
    feats, targs, iters = generate(a.pts, a.steps, a.seed)
    t1 = time.perf_counter()
    ws, info = train(feats, targs, epochs=a.epochs)
    t2 = time.perf_counter()
    os.makedirs(os.path.dirname(a.out), exist_ok=True)
    ws.save(a.out)
    info.update({"solve_iters": iters, "t_generate_s": round(t1 - t0, 1), "t_train_s": round(t2 - t1, 1),
                 "out": a.out})
    print(json.dumps(info), flush=True)


if __name__ == "__main__":
    main()
