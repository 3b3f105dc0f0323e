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
