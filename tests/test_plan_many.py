"""Host plans of many scenes on a thread pool (fastmbcui_b200.plan_many):
identical to planning the scenes one by one (ordering, pattern, supernodes),
whatever the number of threads each plan uses, and faster than planning
them one by one on one thread, on a multi-core host."""
import os
import time

import numpy as np

import fastmbcui_b200 as F
from fastmbcui_b200 import scenes as S


def _same(a, b):
    assert np.array_equal(a.order()[0], b.order()[0])
    assert np.array_equal(a.order()[1], b.order()[1])
    for x, y in zip(a.pattern(), b.pattern()):
        assert np.array_equal(x, y)
    for x, y in zip(a.supernodes(), b.supernodes()):
        assert np.array_equal(x, y)


def test_plan_many_matches_serial_plans():
    scs = S.uneven_batch(6, first_seed=3)
    specs = [(sc.y, sc.rho, sc.lam, sc.max_super) for sc in scs]
    t0 = time.perf_counter()
    serial = [F.Plan(*a, n_threads=1) for a in specs]
    t_serial = time.perf_counter() - t0
    t0 = time.perf_counter()
    many = F.plan_many(specs)
    t_many = time.perf_counter() - t0
    assert len(many) == len(serial)
    for a, b in zip(serial, many):
        _same(a, b)
    if (os.cpu_count() or 1) >= 4:
        # several plans at once; generous bound for a loaded host
        assert t_many < 0.9 * t_serial, (t_many, t_serial)
    assert F.plan_many([]) == []
