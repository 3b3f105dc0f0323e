"""Product host plan (libmbc.so, C ABI) equals the oracle bit for bit."""
import numpy as np
import pytest

import fastmbcui_b200 as F
import oracle as O
from fastmbcui_b200 import scenes as S

KEYS = [("order", ("P", "scale")), ("pattern", ("ptr", "ind")),
        ("supernodes", ("sup_ptr", "sup_ind", "sup_parent")), ("factor_pattern", ("lptr", "lind"))]


def assert_same(y, rho=3.0, lam=1.5, max_super=2048):
    p = F.Plan(y, rho, lam, max_super)
    o = O.plan(y, rho, lam, max_super)
    for meth, names in KEYS:
        got = getattr(p, meth)()
        for g, k in zip(got, names):
            assert np.array_equal(g, o[k]), (meth, k)
    assert p.info.n_super == o["n_super"]
    assert p.info.theta_nnz == int(o["th_ptr"][-1])
    # the row-wise view the preconditioner's gather walks (built by a
    # parallel transpose): per row, the columns ascending, as a stable
    # counting sort of lind gives
    rp, rc, rm = p.factor_rows()
    lptr, lind = np.asarray(o["lptr"]), np.asarray(o["lind"], np.int64)
    n = len(lptr) - 1
    order = np.argsort(lind, kind="stable")
    assert np.array_equal(rm, order)
    assert np.array_equal(rc, np.repeat(np.arange(n), np.diff(lptr))[order])
    assert np.array_equal(rp, np.concatenate([[0], np.cumsum(np.bincount(lind, minlength=n))]))
    return p, o


@pytest.mark.parametrize("seed", range(6))
def test_random_ellipsoid_scenes(seed):
    rng = np.random.default_rng(seed)
    nb = int(rng.integers(1, 5))
    sc = S.ellipsoids_scene(nb, rng.integers(200, 1500, size=nb), seed=100 + seed)
    assert_same(sc.y)


@pytest.mark.parametrize("rho", [1.15, 1.2, 2.0, 3.0, 4.0, 6.9, 7.0, 9.5])
def test_rho_branches_and_float_widening(rho):
    sc = S.coins_scene(n_coins=2, pts=700)
    assert_same(sc.y, rho=rho)


@pytest.mark.parametrize("max_super", [1, 2, 5, 17])
def test_supernode_cap(max_super):
    sc = S.sphere_scene(subdiv=3)
    p, _ = assert_same(sc.y, max_super=max_super)
    sp, _, _ = p.supernodes()
    assert np.diff(sp).max() <= max_super


@pytest.mark.parametrize("lam", [1.0, 1.5, 3.0])
def test_lambda(lam):
    assert_same(S.ellipsoids_scene(2, 600, seed=5).y, lam=lam)


def test_sphere_and_ties():
    assert_same(S.sphere_scene().y)
    g = np.stack(np.meshgrid(np.arange(10), np.arange(10), np.arange(4)), -1).reshape(-1, 3) * 0.25
    assert_same(g.astype(np.float64))


def test_far_apart_clusters():
    rng = np.random.default_rng(3)
    a = np.float32(rng.random((300, 3))).astype(np.float64)
    y = np.concatenate([a, a + 1000.0, a * 0.01 - 50.0])
    assert_same(y)


def test_two_points():
    assert_same(np.array([[0.0, 0, 0], [0.5, -1.0, 2.0]]))


def test_large_scene_plan():
    sc = S.ellipsoids_scene(32, 2000, seed=4)
    p, _ = assert_same(sc.y)
    assert p.info.n == 64000


def test_errors():
    with pytest.raises(F.MbcError) as e:
        F.Plan(np.zeros((1, 3)))
    assert e.value.status == 8  # MBC_COVERAGE: the reference asserts here
    with pytest.raises(F.MbcError):
        F.Plan(np.array([[0.0, 0, 0], [1.0, 0, 0], [1.0, 0, 0], [0, 1.0, 0]]))
    with pytest.raises(F.MbcError) as e:
        F.Plan(np.array([[0.0, np.nan, 0], [1.0, 0, 0]]))
    assert e.value.status == 4
    with pytest.raises(F.MbcError):
        F.Plan(np.zeros((0, 3)))
    with pytest.raises(F.MbcError):
        F.Plan(np.random.default_rng(0).random((10, 3)), rho=-1.0)


def test_boxes_above_floor_plan():
    """The large configuration (N = 200000, rho 4, supernodes capped at 512):
    the floor's 400 x 250 regular grid is full of exactly equal distances, so
    the maximin tie-breaking decides the ordering; the product's plan must
    still equal the oracle's bit for bit."""
    sc = S.large_scene()
    p, _ = assert_same(sc.y, rho=sc.rho, lam=sc.lam, max_super=sc.max_super)
    assert p.info.n == 200000


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
def test_boxes_above_floor_order_matches_reference():
    """On the same points the reference's own maximin ordering and radius
    search (src/maxmin.h, src/nanoflann.hpp built into oracle/_ref) agree
    with the oracle's, at the configuration's rho = 4."""
    sc = S.large_scene()
    P, s = O.order(sc.y)
    Pr, sr = O.ref_order(sc.y)
    assert np.array_equal(P, Pr) and np.array_equal(s, sr)
    ptr, ind = O.pattern(sc.y, P, s, sc.rho)
    ptr2, ind2 = O.ref_pattern(sc.y, Pr, sr, sc.rho)
    assert np.array_equal(ptr, ptr2) and np.array_equal(ind, ind2)


@pytest.mark.parametrize("k", [0, 3])
def test_trajectory32_plan_matches_oracle_and_reference(k):
    """The benchmark's scene (32 ellipsoids x 2000 points on the seed-4
    trajectory, poses 0 and 3): the product's whole plan equals the
    oracle's, and the oracle's ordering and pattern equal the reference's own
    maxmin.h / nanoflann code (oracle/_ref) when it is built."""
    base, q, _ = S.trajectory_scene(32, 2000, seed=4, steps=500)
    sc = S.moved(base, q[k])
    assert_same(sc.y, rho=sc.rho, lam=sc.lam, max_super=sc.max_super)
    if O.ref_available():
        P, s = O.order(sc.y)
        Pr, sr = O.ref_order(sc.y)
        assert np.array_equal(P, Pr) and np.array_equal(s, sr)
        ptr, ind = O.pattern(sc.y, P, s, sc.rho)
        ptr2, ind2 = O.ref_pattern(sc.y, Pr, sr, sc.rho)
        assert np.array_equal(ptr, ptr2) and np.array_equal(ind, ind2)
