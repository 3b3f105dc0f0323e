"""The benchmark's own path at the benchmark's own size.

The 32-ellipsoid trajectory scene (32 ellipsoids x 2000 points, N = Nf =
64000, R = 192 rigid-mode columns, rho 3, lambda 1.5, trajectory seed 4) is
solved by TrajectorySolver exactly as bench.py times it: per step a new host
plan and factor, all 192 columns in one block PCG, warm-started by the
quadratic extrapolation of the previous three steps.  Steps 0-2 build the
history; step 3 is checked.

Checks and their tolerances:
  * every column's FP64 true residual |K^T (f - K x)| / |K^T f| <= 1e-8,
    recomputed by the FP64 CUDA-core kernels (which test_gpu_parity.py pins
    to the oracle at 1e-12);
  * added mass of the 12 columns of two bodies against a tight solve of the
    same columns (plain FP64 method, FP64 CUDA-core matvec, true residual
    <= 1e-12): 1e-6 relative, norm-wise over that block of the tensor;
    forces -Mf a for a unit acceleration of those modes likewise;
  * cold-start iterations of the plain FP64 method on pose 0, against the
    CPU oracle's own PCG on the same columns
    (tests/golden/trajectory32_oracle_iters.json, measured by
    tests/golden/make_trajectory32_oracle_iters.py): within max(3, 3 %) per
    column, or, where the residual lingers near tol so that the crossing
    iteration is ill-determined, an FP64 residual within 1.5 tol after
    exactly the oracle's iteration count.
"""
import json
import os

import numpy as np
import pytest

import fastmbcui_b200 as F
from fastmbcui_b200 import scenes as S
from fastmbcui_b200.trajectory import TrajectorySolver

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "trajectory32_oracle_iters.json")


def _dev(a, dt=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")


class Traj:
    def __init__(self):
        self.base, self.q, _ = S.trajectory_scene(32, 2000, seed=4, steps=500)
        self.scenes = [S.moved(self.base, self.q[k]) for k in range(4)]

    def arrays(self, k):
        sc = self.scenes[k]
        plan = F.Plan(sc.y, sc.rho, sc.lam, sc.max_super)
        return plan, _dev(sc.x), _dev(sc.nx), _dev(sc.y), _dev(sc.rhs())


@pytest.fixture(scope="module")
def traj():
    return Traj()


@pytest.fixture(scope="module")
def stepped(traj):
    ts = TrajectorySolver(traj.base.coef, mode="mixed", fp64_matvec="int8", warm="extrapolate")
    for k in range(3):
        ts.step(*traj.arrays(k))
    plan, x, nx, y, Fd = traj.arrays(3)
    X, st = ts.step(plan, x, nx, y, Fd)
    return plan, x, nx, y, Fd, X, st


def test_bench_step_reaches_fp64_tolerance(traj, stepped):
    plan, x, nx, y, Fd, X, st = stepped
    assert st["n_converged"] == 192, st
    s64 = F.Solver(plan, x=x, nx=nx, y=y, coef=traj.base.coef, precision=F.MBC_F64)  # FP64 CUDA-core matvecs
    F64 = Fd.double()
    b = s64.apply_KT(F64)
    r = s64.apply_KT(F64 - s64.apply_K(X))
    rel = (torch.linalg.norm(r, dim=0) / torch.linalg.norm(b, dim=0)).cpu().numpy()
    assert rel.max() <= 1e-8, (rel.max(), int(rel.argmax()))


def test_bench_step_added_mass_matches_tight_solve(traj, stepped):
    plan, x, nx, y, Fd, X, _ = stepped
    sc = traj.scenes[3]
    cols = list(range(0, 6)) + list(range(6 * 17, 6 * 18))  # bodies 0 and 17
    s64 = F.Solver(plan, x=x, nx=nx, y=y, coef=sc.coef, precision=F.MBC_F64).factor()
    Xt, st = s64.solve(Fd[:, cols].double().contiguous(), X0=X[:, cols].contiguous(), tol=1e-12,
                       max_iters=20000, true_residual=1)
    assert st["true_relres_max"] <= 1.05e-12, st
    w, bp, cen = sc.weights(), sc.body_ptr(), sc.centers
    Mb = s64.added_mass(X[:, cols].contiguous(), w, bp, cen)
    Mt = s64.added_mass(Xt, w, bp, cen)
    err = np.linalg.norm(Mb - Mt) / np.linalg.norm(Mt)
    assert err <= 1e-6, err
    acc = np.ones(len(cols))
    fb, ft = Mb @ acc, Mt @ acc
    assert np.linalg.norm(fb - ft) / np.linalg.norm(ft) <= 1e-6


@pytest.mark.skipif(not os.path.exists(FIXTURE), reason="oracle iteration fixture not generated")
def test_plain_fp64_iterations_match_oracle(traj):
    with open(FIXTURE) as f:
        ref = json.load(f)
    plan, x, nx, y, Fd = traj.arrays(0)
    cols = ref["columns"]
    s64 = F.Solver(plan, x=x, nx=nx, y=y, coef=traj.base.coef, precision=F.MBC_F64).factor()
    # the batched PCG runs every column's own recurrence (the per-RHS loop's,
    # with shared matvec launches): its iterations are the per-column ones
    _, st, its = s64.solve(Fd[:, cols].double().contiguous(), tol=ref["tol"], max_iters=5000, iters=True)
    b = s64.apply_KT(Fd.double())
    for c, got, want in zip(cols, its, ref["iters"]):
        if abs(int(got) - want) <= max(3, 0.03 * want):
            continue
        # a residual that lingers just above tol makes the crossing iteration
        # ill-determined: then, after exactly the oracle's iteration count,
        # the column's FP64 residual must be within 1.5 tol
        Xc, _ = s64.solve(Fd[:, c].double().contiguous(), tol=ref["tol"], max_iters=want)
        r = s64.apply_KT(Fd[:, c].double() - s64.apply_K(Xc))
        rel = float(torch.linalg.norm(r) / torch.linalg.norm(b[:, c]))
        assert rel <= 1.5 * ref["tol"], (c, int(got), want, rel)
