"""The CPU oracle is pinned to the reference's own code.

Golden fixtures (tests/golden/plan_*.npz) hold the reference's maximin
ordering and kd-tree pattern (src/maxmin.h, src/nanoflann.hpp compiled by
oracle/Makefile) on seeded scenes; the oracle must reproduce them and the
supernodes derived from them.  When oracle/_ref/libref.so is present the
reference code is also run live on further scenes.
"""
import glob
import os

import numpy as np
import pytest

import oracle as O
from fastmbcui_b200 import scenes as S

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "plan_*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_oracle_matches_golden(path):
    g = np.load(path)
    y = g["y"].astype(np.float64)
    pl = O.plan(y, float(g["rho"]), float(g["lam"]), int(g["max_super"]))
    for k in ("P", "scale", "ptr", "ind", "sup_ptr", "sup_ind", "sup_parent", "lptr", "lind"):
        assert np.array_equal(pl[k], g[k]), k


def _clouds():
    rng = np.random.default_rng(7)
    yield "cube", np.float32(rng.random((1500, 3)) * 2 - 1).astype(np.float64)
    t = rng.random(1200) * 2 * np.pi
    u = rng.random(1200) * 2 * np.pi
    torus = np.stack([(1 + 0.3 * np.cos(u)) * np.cos(t), (1 + 0.3 * np.cos(u)) * np.sin(t), 0.3 * np.sin(u)], 1)
    yield "torus", np.float32(torus).astype(np.float64)
    g = np.stack(np.meshgrid(np.arange(12), np.arange(12), np.arange(3)), -1).reshape(-1, 3) * 0.1
    yield "lattice_ties", g.astype(np.float64)
    yield "two", np.array([[0.0, 0, 0], [1.0, 2.0, 3.0]])
    yield "ellipsoids", S.ellipsoids_scene(2, 900, seed=3).y


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("rho", [1.15, 3.0, 7.5])
def test_oracle_matches_reference_live(rho):
    for name, y in _clouds():
        P, s = O.order(y)
        Pr, sr = O.ref_order(y)
        assert np.array_equal(P, Pr) and np.array_equal(s, sr), name
        ptr, ind = O.pattern(y, P, s, rho)
        ptr2, ind2 = O.ref_pattern(y, Pr, sr, rho)
        assert np.array_equal(ptr, ptr2) and np.array_equal(ind, ind2), name


def test_oracle_single_point_fails_like_reference():
    # one point: its length scale is 0, the diagonal predicate 0 < 0 fails and
    # aggregation cannot cover the point (preprocess.h:593 asserts)
    with pytest.raises(RuntimeError):
        O.plan(np.zeros((1, 3)))


def test_oracle_duplicate_points_fail_coverage():
    y = np.array([[0.0, 0, 0], [1.0, 0, 0], [1.0, 0, 0], [0, 1.0, 0]])
    with pytest.raises(RuntimeError):
        O.plan(y)
