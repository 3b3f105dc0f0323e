"""Several independent scenes: concurrent solves (one stream and host thread
each) and CUDA-graph replay of the PCG iteration blocks must give bitwise the
results of plain one-by-one solves (every reduction runs in a fixed order)."""
import numpy as np
import pytest

import fastmbcui_b200 as F
from fastmbcui_b200 import scenes as S

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _t(a, dt=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")


@pytest.fixture(scope="module")
def batch():
    scs = [S.ellipsoids_scene(nb, pts, seed=s) for nb, pts, s in ((1, 1500, 40), (3, 900, 41), (2, 1200, 42))]
    out = []
    for sc in scs:
        plan = F.Plan(sc.y, sc.rho, sc.lam, sc.max_super)
        out.append((sc, plan))
    return out


def _solver(sc, plan, prec):
    return F.Solver(plan, x=_t(sc.x), nx=_t(sc.nx), y=_t(sc.y), coef=sc.coef, precision=prec)


@pytest.mark.parametrize("prec", [F.MBC_F32, F.MBC_F64])
def test_concurrent_and_graph_solves_equal_sequential(batch, prec):
    dt = torch.float64 if prec == F.MBC_F64 else torch.float32
    opts = dict(out_dtype=torch.float64, tol=1e-8, max_iters=3000)
    seq = []
    for sc, plan in batch:
        s = _solver(sc, plan, prec).factor()
        seq.append(s.solve(_t(sc.rhs(), dt), **opts))
    torch.cuda.synchronize()
    for graph in (0, 1):
        solvers = [_solver(sc, plan, prec) for sc, plan in batch]
        Fs = [_t(sc.rhs(), dt) for sc, _ in batch]
        res = F.solve_many(solvers, Fs, graph=graph, **opts)
        for (X, st), (Xs, sts) in zip(res, seq):
            assert st["n_converged"] == sts["n_converged"] and st["iters_max"] == sts["iters_max"]
            assert torch.equal(X, Xs), graph
            assert st["true_relres_max"] <= 1e-8 or prec == F.MBC_F64
