"""Column compaction of the batched PCG (mbc_solve_options.compact) on the
GPU: once at most half of the columns still iterate, the solve continues on
those alone.  Compaction changes no column's recurrence, only which columns
the kernels carry, so the result must match the uncompacted solve:
iterations within 2 per column (the per-column dot products are grouped
differently at another width), fitted flux within 1e-8 of |F|, FP64 true
residual <= 1.05e-8 per column.  Also with the INT8 FP64 matvec (its
restarted columns).
"""
import numpy as np
import pytest

import fastmbcui_b200 as F
import oracle as O
from fastmbcui_b200 import scenes as S

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _dev(a, dt=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")


@pytest.mark.parametrize("fp64_matvec", ["simt", "int8"])
def test_compacted_solve_matches(fp64_matvec):
    sc = S.ellipsoids_scene(3, 1000, seed=17)
    plan = F.Plan(sc.y, sc.rho, sc.lam, sc.max_super)
    s = F.Solver(plan, x=_dev(sc.x), nx=_dev(sc.nx), y=_dev(sc.y), coef=sc.coef, precision=F.MBC_F64)
    s.set_fp64_matvec(fp64_matvec).factor()
    Fm = sc.rhs()
    X0, st0, it0 = s.solve(_dev(Fm, torch.float64), tol=1e-8, max_iters=3000, check_every=4, iters=True)
    X1, st1, it1 = s.solve(_dev(Fm, torch.float64), tol=1e-8, max_iters=3000, check_every=4, compact=1,
                           iters=True)
    X0, X1 = X0.cpu().numpy(), X1.cpu().numpy()
    assert np.abs(it1 - it0).max() <= 2 + (8 if fp64_matvec == "int8" else 0), (it0, it1)
    op = O.Op.from_scene(sc)
    b = op.KT(Fm)
    rel = np.linalg.norm(op.KT(Fm - op.K(X1)), axis=0) / np.linalg.norm(b, axis=0)
    assert rel.max() <= 1.05e-8, rel
    assert np.linalg.norm(op.K(X1) - op.K(X0)) / np.linalg.norm(Fm) < 1e-8


def test_compacted_polish_of_the_mixed_solve():
    """MBC_F32 solves: the FP64 polish compacts too; every column still ends
    at an FP64 true residual <= 1.05e-8, and the flux matches the
    uncompacted solve within 1e-7 of |F|."""
    sc = S.ellipsoids_scene(3, 1000, seed=17)
    plan = F.Plan(sc.y, sc.rho, sc.lam, sc.max_super)
    s = F.Solver(plan, x=_dev(sc.x), nx=_dev(sc.nx), y=_dev(sc.y), coef=sc.coef, precision=F.MBC_F32).factor()
    Fm = sc.rhs()
    X0, _ = s.solve(_dev(Fm), out_dtype=torch.float64, tol=1e-8, max_iters=3000, check_every=4)
    X1, st1 = s.solve(_dev(Fm), out_dtype=torch.float64, tol=1e-8, max_iters=3000, check_every=4, compact=1)
    X0, X1 = X0.cpu().numpy(), X1.cpu().numpy()
    op = O.Op.from_scene(sc)
    b = op.KT(Fm)
    rel = np.linalg.norm(op.KT(Fm - op.K(X1)), axis=0) / np.linalg.norm(b, axis=0)
    assert rel.max() <= 1.05e-8, (rel, st1)
    assert np.linalg.norm(op.K(X1) - op.K(X0)) / np.linalg.norm(Fm) < 1e-7
