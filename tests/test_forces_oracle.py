"""Added mass of the solved strengths (the observable downstream of the solve),
CPU oracle against closed forms.

* Unit sphere (icosphere subdivision 4): M = (2/3) pi rho R^3 on the
  translation block, 0 on the rotation block (Lamb, Hydrodynamics, sect. 92).
* Single ellipsoid (Fibonacci points with exact area weights, sources 0.15
  inside): translation added masses rho V alpha0 / (2 - alpha0) along the
  principal axes, alpha0 = abc int_0^inf dl / ((a^2+l) Delta(l)),
  Delta(l) = sqrt((a^2+l)(b^2+l)(c^2+l)) (Lamb, sect. 114); measured
  agreement ~2e-5, asserted at 2e-4.
"""
import numpy as np
import pytest

import oracle as O
from fastmbcui_b200 import scenes as S


def _solve(sc, cols, tol):
    op = O.Op.from_scene(sc)
    pl = O.plan(sc.y, sc.rho, sc.lam, sc.max_super)
    _, lval, _ = O.factor(op, pl)
    Fm = sc.rhs()
    X = np.zeros((sc.n, Fm.shape[1]))
    Xc, _ = O.solve(op, pl, lval, Fm[:, cols], maxits=3000, tol=tol)
    X[:, cols] = Xc
    return X


def test_sphere_added_mass_closed_form():
    sc = S.sphere_scene()
    # rotation modes have zero normal velocity on a sphere centred at 0
    X = _solve(sc, [0, 1, 2], 1e-10)
    Mf = O.added_mass(sc, X, rho_f=1.0)
    m = 2.0 / 3.0 * np.pi
    assert np.allclose(np.diag(Mf)[:3], m, rtol=2e-3), np.diag(Mf)
    off = Mf.copy()
    off[[0, 1, 2], [0, 1, 2]] = 0.0
    assert np.abs(off).max() < 1e-3 * m


def _lamb_translation(a, b, c):
    from scipy.integrate import quad

    def alpha(p, q, r):
        f = lambda l: 1.0 / ((p * p + l) * np.sqrt((p * p + l) * (q * q + l) * (r * r + l)))
        return p * q * r * quad(f, 0, np.inf, limit=200)[0]

    V = 4.0 / 3.0 * np.pi * a * b * c
    out = []
    for p, q, r in ((a, b, c), (b, c, a), (c, a, b)):
        a0 = alpha(p, q, r)
        out.append(V * a0 / (2.0 - a0))
    return np.array(out)


@pytest.mark.parametrize("axes", [(1.2, 0.8, 0.6), (1.4, 1.0, 0.5)])
def test_ellipsoid_added_mass_vs_lamb(axes):
    pytest.importorskip("scipy")
    sc = S.ellipsoid_fibonacci_scene(axes, 2000, offset=0.15)
    X = _solve(sc, [0, 1, 2], 1e-10)
    Mf = O.added_mass(sc, X, rho_f=1.0)
    want = _lamb_translation(*axes)
    assert np.allclose(np.diag(Mf)[:3], want, rtol=2e-4), (np.diag(Mf)[:3], want)
    # principal axes: the off-diagonal translation entries vanish, and the
    # translation-rotation coupling of a centred ellipsoid is zero
    T = Mf[:3, :3]
    assert np.abs(T - np.diag(np.diag(T))).max() < 1e-4 * want.max()
    assert np.abs(Mf[3:, :3]).max() < 1e-4 * want.max()


def test_added_mass_is_linear_in_strengths():
    sc = S.ellipsoids_scene(2, [300, 400], seed=5)
    rng = np.random.default_rng(0)
    X1, X2 = rng.standard_normal((sc.n, 3)), rng.standard_normal((sc.n, 3))
    a = O.added_mass(sc, X1)
    b = O.added_mass(sc, X2)
    c = O.added_mass(sc, 2.0 * X1 - X2)
    assert np.allclose(c, 2.0 * a - b, rtol=1e-12, atol=1e-12 * np.abs(c).max())
