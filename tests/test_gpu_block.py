"""Block PCG (mbc_solve_options.schedule = MBC_SCHED_BLOCK) on the GPU.

The block recursion shares one Krylov space over the columns; each column
still stops on its own residual, so the result must satisfy the same
criterion as the batched per-column PCG:
  * every column's FP64 true residual |K^T (f - K x)| / |K^T f| <= tol,
    recomputed with the FP64 CUDA-core kernels (pinned to the oracle);
  * the fitted flux K x within 1e-6 of the batched solve's, relative to |F|;
  * the longest column takes no more iterations than in the batched solve
    plus one check block (the shared space only adds directions);
with the FP64 factor and FP64 matvec, with the FP32 factor and the INT8
FP64 matvec, from warm starts, and with right-hand-side columns that are
zero (the rotational modes of a sphere).
"""
import numpy as np
import pytest

import fastmbcui_b200 as F
from fastmbcui_b200 import scenes as S

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dev(a, dt=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")


def _case(sc):
    plan = F.Plan(sc.y, sc.rho, sc.lam, sc.max_super)
    return plan, _dev(sc.x), _dev(sc.nx), _dev(sc.y), _dev(sc.rhs(), torch.float64)


def _true_rel(plan, x, nx, y, coef, Fd, X):
    s = F.Solver(plan, x=x, nx=nx, y=y, coef=coef, precision=F.MBC_F64)
    b = s.apply_KT(Fd)
    r = s.apply_KT(Fd - s.apply_K(X))
    nb = torch.linalg.norm(b, dim=0)
    rel = torch.where(nb > 0, torch.linalg.norm(r, dim=0) / torch.clamp(nb, min=1e-300), torch.zeros_like(nb))
    return rel.cpu().numpy(), s


@pytest.mark.parametrize("mode", ["fp64-simt", "mixed-int8"])
def test_block_matches_batched(mode):
    sc = S.ellipsoids_scene(3, 1000, seed=17)
    plan, x, nx, y, Fd = _case(sc)
    prec = F.MBC_F64 if mode == "fp64-simt" else F.MBC_F32
    mv = "simt" if mode == "fp64-simt" else "int8"
    s = F.Solver(plan, x=x, nx=nx, y=y, coef=sc.coef, precision=prec).set_fp64_matvec(mv).factor()
    opts = dict(out_dtype=torch.float64, tol=1e-8, max_iters=4000, iters=True, fp64_recursion=1)
    Xb, stb, itb = s.solve(Fd, schedule=F.MBC_SCHED_BATCHED, **opts)
    Xk, stk, itk = s.solve(Fd, schedule=F.MBC_SCHED_BLOCK, **opts)
    assert stk["n_converged"] == Fd.shape[1], stk
    rel, s64 = _true_rel(plan, x, nx, y, sc.coef, Fd, Xk)
    assert rel.max() <= 1e-8, rel
    flux = torch.linalg.norm(s64.apply_K(Xk) - s64.apply_K(Xb)) / torch.linalg.norm(Fd)
    assert float(flux) < 1e-6
    assert itk.max() <= itb.max() + 8, (itk.max(), itb.max())


def test_block_warm_start_and_zero_columns():
    sc = S.sphere_scene(subdiv=3)  # rotational right-hand sides of a sphere are zero
    plan, x, nx, y, Fd = _case(sc)
    s = F.Solver(plan, x=x, nx=nx, y=y, coef=sc.coef, precision=F.MBC_F64).factor()
    X, st, it = s.solve(Fd, tol=1e-10, max_iters=4000, iters=True, schedule=F.MBC_SCHED_BLOCK)
    zero = (torch.linalg.norm(Fd, dim=0) == 0).cpu().numpy()
    assert zero.any() and np.all(it[zero] == 0)
    assert torch.all(X[:, torch.as_tensor(zero, device="cuda")] == 0)
    rel, _ = _true_rel(plan, x, nx, y, sc.coef, Fd, X)
    assert rel.max() <= 1e-10, rel
    # from a perturbed start the block recursion still ends at the tolerance
    g = torch.Generator(device="cuda").manual_seed(0)
    X0 = X * (1.0 + 1e-3 * torch.randn(X.shape, generator=g, device="cuda", dtype=X.dtype))
    X2, st2, it2 = s.solve(Fd, X0=X0, tol=1e-10, max_iters=4000, iters=True, schedule=F.MBC_SCHED_BLOCK)
    rel2, _ = _true_rel(plan, x, nx, y, sc.coef, Fd, X2)
    assert rel2.max() <= 1e-10 and st2["n_converged"] == Fd.shape[1]
    assert it2.max() < it.max()
