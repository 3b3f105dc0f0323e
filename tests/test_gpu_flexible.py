"""Flexible CG in FP64 around the FP32 solver's plain PCG (tensor-core matvec)
on the GPU, against the FP64 oracle and the FP64 batched solve.

Tolerances: FP64 true relative normal-equation residual <= 1.05e-8 per column
(oracle-recomputed), fitted flux within 1e-6 of the FP64 solve's (relative to
|f|); and at most a third as many FP64 operator applications as the FP64
PCG's iterations."""
import numpy as np
import pytest

import fastmbcui_b200 as F
import oracle as O
from fastmbcui_b200 import scenes as S
from fastmbcui_b200.flexible import solve_flexible

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _t(a, dt=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")


def test_flexible_solve_matches_fp64_with_few_fp64_applies():
    sc = S.ellipsoids_scene(2, 1500, seed=21)
    plan = F.Plan(sc.y, sc.rho, sc.lam, sc.max_super)
    x, nx, y = _t(sc.x), _t(sc.nx), _t(sc.y)
    s64 = F.Solver(plan, x=x, nx=nx, y=y, coef=sc.coef, precision=F.MBC_F64).factor()
    s32 = F.Solver(plan, x=x, nx=nx, y=y, coef=sc.coef, precision=F.MBC_F32).factor()
    Fm = sc.rhs()
    X, info = solve_flexible(s64, s32, _t(Fm), tol=1e-8, inner_iters=40)
    assert info["converged"] == Fm.shape[1], info
    X = X.cpu().numpy()
    op = O.Op.from_scene(sc)
    b = op.KT(Fm)
    rel = np.linalg.norm(op.KT(Fm - op.K(X)), axis=0) / np.linalg.norm(b, axis=0)
    assert rel.max() <= 1.05e-8, rel
    X64, st64 = s64.solve(_t(Fm, torch.float64), tol=1e-8, max_iters=4000)
    d = np.linalg.norm(op.K(X) - op.K(X64.cpu().numpy())) / np.linalg.norm(Fm)
    assert d < 1e-6, d
    assert 3 * info["fp64_applies"] <= st64["iters_max"], (info, st64["iters_max"])
