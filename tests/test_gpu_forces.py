"""Added mass and fluid forces on the GPU (mbc_added_mass) against the FP64 oracle.

Tolerances:
  * the reduction itself (GPU on the oracle's strengths): 1e-11 relative;
  * end to end (GPU solve to 1e-8, FP32 mixed or FP64 plain, then the
    added mass) against the oracle's FP64 solve to 1e-12: 1e-6 relative
    (norm-wise over the tensor), forces -Mf a likewise;
  * unit sphere: (2/3) pi on the translation block within 2e-3.
"""
import numpy as np
import pytest

import fastmbcui_b200 as F
import oracle as O
from fastmbcui_b200 import _lib
from fastmbcui_b200 import scenes as S

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _dev(a, dt=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


class Case:
    def __init__(self, sc):
        self.sc = sc
        self.op = O.Op.from_scene(sc)
        self.pl = O.plan(sc.y, sc.rho, sc.lam, sc.max_super)
        _, self.lval, _ = O.factor(self.op, self.pl)
        self.plan = F.Plan(sc.y, sc.rho, sc.lam, sc.max_super)
        self.x, self.nx, self.y = _dev(sc.x), _dev(sc.nx), _dev(sc.y)
        Fm = sc.rhs()
        self.Fm = Fm
        self.cols = [c for c in range(Fm.shape[1]) if np.linalg.norm(Fm[:, c]) > 0]
        X = np.zeros((sc.n, Fm.shape[1]))
        X[:, self.cols], _ = O.solve(self.op, self.pl, self.lval, Fm[:, self.cols], maxits=4000, tol=1e-12)
        self.X = X
        self.Mf = O.added_mass(sc, X)

    def solver(self, prec):
        return F.Solver(self.plan, x=self.x, nx=self.nx, y=self.y, coef=self.sc.coef, precision=prec).factor()

    def gpu_added_mass(self, s, X, accel=None):
        return s.added_mass(X, self.sc.weights(), self.sc.body_ptr(), self.sc.centers, 1.0, accel=accel)


@pytest.fixture(scope="module")
def ells():
    return Case(S.ellipsoids_scene(2, 1500, seed=21))


@pytest.fixture(scope="module")
def fib():
    return Case(S.ellipsoid_fibonacci_scene((1.2, 0.8, 0.6), 2000, offset=0.15))


def test_reduction_matches_oracle(ells):
    s = ells.solver(F.MBC_F64)
    Mf = ells.gpu_added_mass(s, _dev(ells.X, torch.float64))
    assert rel(Mf, ells.Mf) < 1e-11


@pytest.mark.parametrize("prec", [F.MBC_F32, F.MBC_F64])
@pytest.mark.parametrize("case", ["ells", "fib"])
def test_added_mass_and_forces_end_to_end(case, prec, request):
    c = request.getfixturevalue(case)
    s = c.solver(prec)
    X, st = s.solve(_dev(c.Fm, torch.float64), out_dtype=torch.float64, tol=1e-8, max_iters=4000)
    assert st["n_converged"] == c.Fm.shape[1]
    a = np.random.default_rng(7).standard_normal(c.Fm.shape[1])
    Mf, f = c.gpu_added_mass(s, X, accel=a)
    assert rel(Mf, c.Mf) < 1e-6, rel(Mf, c.Mf)
    assert rel(f, -c.Mf @ a) < 1e-6


def test_sphere_closed_form():
    sc = S.sphere_scene()
    plan = F.Plan(sc.y, sc.rho, sc.lam, sc.max_super)
    s = F.Solver(plan, x=_dev(sc.x), nx=_dev(sc.nx), y=_dev(sc.y), coef=sc.coef, precision=F.MBC_F32).factor()
    X, st = s.solve(_dev(sc.rhs()[:, :3]), out_dtype=torch.float64, tol=1e-10, max_iters=4000)
    Mf = s.added_mass(X, sc.weights(), sc.body_ptr(), sc.centers, 1.0)
    assert np.allclose(np.diag(Mf[:3, :3]), 2.0 / 3.0 * np.pi, rtol=2e-3)


def test_argument_errors(ells):
    s = ells.solver(F.MBC_F64)
    X = _dev(ells.X, torch.float64)
    with pytest.raises(_lib.MbcError, match="body_ptr"):
        s.added_mass(X, ells.sc.weights(), np.array([0, 5000, 10], np.int32), ells.sc.centers)
    with pytest.raises(_lib.MbcError, match="R == 6"):
        s.added_mass(X[:, :5], ells.sc.weights(), ells.sc.body_ptr(), ells.sc.centers, accel=np.zeros(5))
    Kd = ells.sc.dense_K().astype(np.float32)
    sd = F.Solver(ells.plan, M=_dev(Kd), precision=F.MBC_F64)
    with pytest.raises(_lib.MbcError, match="point-kernel"):
        sd.added_mass(X, ells.sc.weights(), ells.sc.body_ptr(), ells.sc.centers)
