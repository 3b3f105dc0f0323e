"""Reusing a trajectory step's plan (ordering, pattern, supernodes) for later
steps, with the factor rebuilt on the current geometry (the opt-in
``--plan-every`` mode of the benchmark): the oracle's FP64 PCG still reaches
the tolerance, and after 10 steps of motion it needs at most 10 % more
iterations than with a fresh plan (measured 0-3 %)."""
import numpy as np

import oracle as O
from fastmbcui_b200 import scenes as S


def test_stale_plan_after_ten_steps():
    base, q, _ = S.trajectory_scene(6, 1000, seed=3, steps=12)
    stale = O.plan(S.moved(base, q[0]).y, 3.0)
    sc = S.moved(base, q[10])
    op = O.Op.from_scene(sc)
    fresh = O.plan(sc.y, 3.0)
    assert not np.array_equal(fresh["P"], stale["P"])  # the ordering did change
    for c in (0, 7):
        its = []
        for pl in (fresh, stale):
            _, lval, _ = O.factor(op, pl)
            _, it, rr = O.pcg(op, pl, lval, f=sc.rhs()[:, c], maxits=3000, tol=1e-8)
            assert rr < 1e-8
            its.append(it)
        assert its[1] <= 1.1 * its[0], its


def test_trajectory_solver_plan_every():
    """TrajectorySolver.plan_for: a new plan every plan_every calls (1 = every
    call, the plain method), the same object in between."""
    import fastmbcui_b200 as F
    from fastmbcui_b200 import scenes as S
    from fastmbcui_b200.trajectory import TrajectorySolver

    sc = S.ellipsoids_scene(2, 300, seed=1)
    ts = TrajectorySolver(sc.coef, plan_every=3)
    plans = [ts.plan_for(sc.y, sc.rho, sc.lam, sc.max_super) for _ in range(7)]
    assert plans[0] is plans[1] is plans[2] and plans[3] is plans[4] is plans[5] and plans[6] is not plans[5]
    assert plans[3] is not plans[0]
    ts1 = TrajectorySolver(sc.coef)
    a, b = ts1.plan_for(sc.y, sc.rho, sc.lam, sc.max_super), ts1.plan_for(sc.y, sc.rho, sc.lam, sc.max_super)
    assert a is not b
    P0, _ = a.order()
    assert np.array_equal(P0, F.Plan(sc.y, sc.rho, sc.lam, sc.max_super).order()[0])
