"""Synthetic scene generators and the warm-start plumbing (host side)."""
import numpy as np

from fastmbcui_b200 import scenes as S
from fastmbcui_b200 import warmstart as W


def test_ellipsoid_area_closed_forms():
    assert abs(S.ellipsoid_area((1, 1, 1)) / (4 * np.pi) - 1) < 1e-6
    # prolate spheroid a > b = c: 2 pi b^2 (1 + a / (b e) asin e)
    a, b = 2.0, 1.0
    e = np.sqrt(1 - b * b / (a * a))
    want = 2 * np.pi * b * b * (1 + a / (b * e) * np.arcsin(e))
    assert abs(S.ellipsoid_area((a, b, b)) / want - 1) < 1e-6


def test_weights_and_body_offsets():
    sc = S.ellipsoids_scene(3, [400, 700, 900], seed=11)
    ptr = sc.body_ptr()
    assert list(ptr) == [0, 400, 1100, 2000]
    w = sc.weights().astype(np.float64)
    for b in range(3):
        assert abs(w[ptr[b]:ptr[b + 1]].sum() / sc.meta["areas"][b] - 1) < 1e-6
    fib = S.ellipsoid_fibonacci_scene((1.2, 0.8, 0.6), 1000)
    assert abs(fib.weights().astype(np.float64).sum() / fib.meta["areas"][0] - 1) < 1e-4


def test_rigid_move_preserves_shapes():
    base, q, _ = S.trajectory_scene(4, 200, seed=2, steps=20)
    sc = S.moved(base, q[13])
    for b in range(4):
        r = sc.row_body == b
        d0 = np.linalg.norm(base.x[r][:, None] - base.x[r][None], axis=-1)
        d1 = np.linalg.norm(sc.x[r][:, None] - sc.x[r][None], axis=-1)
        assert np.abs(d0 - d1).max() < 1e-5
        # normals stay unit and the sources keep their depth below the surface
        assert np.allclose(np.linalg.norm(sc.nx[r], axis=1), 1.0, atol=1e-6)
        s = sc.src_body == b
        assert np.allclose(np.linalg.norm(sc.x[r] - sc.y[s], axis=1), 0.05, atol=1e-5)
    assert np.allclose(sc.centers, base.centers + q[13, :, :3], atol=1e-5)


def test_trajectory_keeps_bodies_apart():
    base, q, _ = S.trajectory_scene(32, 50, seed=4, steps=500)
    rmax = base.meta["axes"].max(axis=1)
    for k in range(0, 500, 25):
        c = base.centers + q[k, :, :3]
        d = np.linalg.norm(c[:, None] - c[None], axis=-1) + np.eye(32) * 1e9
        assert (d - rmax[:, None] - rmax[None]).min() > 0


def test_neighbour_pairs_and_features():
    rng = np.random.default_rng(0)
    cen = rng.random((12, 3)) * 10
    pairs = W.neighbour_pairs(cen, k=8)
    assert pairs.shape == (12 * 9, 2)
    for b in range(12):
        blk = pairs[9 * b:9 * b + 9]
        assert blk[0, 0] == b and np.all(blk[:, 1] == b)  # itself first
        d = np.linalg.norm(cen - cen[b], axis=1)
        assert set(blk[1:, 0]) == set(np.argsort(d, kind="stable")[1:9])
    base, q, _ = S.trajectory_scene(6, 100, seed=1, steps=3)
    p = W.neighbour_pairs(base.centers)
    f = W.pair_features(p, q[0], q[1], base.centers, base.meta["axes"], base.meta["rot"])
    g = W.cold_features(p, q[1], base.centers, base.meta["axes"], base.meta["rot"])
    assert f.shape == (len(p), W.N_FEATURES) and g.shape == (len(p), W.N_COLD_FEATURES)
    assert np.isfinite(f).all() and np.isfinite(g).all()
    # the self flag marks exactly the diagonal pairs
    assert np.array_equal(g[:, 5] == 1.0, p[:, 0] == p[:, 1])


def test_large_scene_geometry():
    """The large configuration: 20 boxes + floor, N = Nf = 200000, R = 120
    (the floor is static), sources inside the boxes and below the floor,
    bodies clear of one another and of the floor."""
    sc = S.large_scene()
    assert sc.n == sc.nf == 200000 and sc.n_bodies == 21
    assert sc.rho == 4.0 and sc.max_super == 512
    F = sc.rhs()
    assert F.shape == (200000, 120)
    floor_rows = sc.row_body == 20
    assert floor_rows.sum() == 100000 and np.all(F[floor_rows] == 0)
    # every box row has a nonzero translation column of its own box
    assert np.all(np.abs(F[~floor_rows]).max(axis=1) > 0)
    # floor sources below the patch, box sources strictly inside their box
    assert np.all(sc.y[sc.src_body == 20, 2] < 0) and np.all(sc.x[floor_rows, 2] == 0)
    sides = sc.meta["sides"]
    for b in range(20):
        pts = sc.x[sc.row_body == b] - sc.centers[b]
        src = sc.y[sc.src_body == b] - sc.centers[b]
        # the rotation is unknown here: compare distances to the centre
        assert np.linalg.norm(src, axis=1).max() < np.linalg.norm(pts, axis=1).max()
        assert np.linalg.norm(pts, axis=1).max() <= sides[b] * np.sqrt(3) / 2 + 1e-5
        assert (sc.x[sc.row_body == b, 2]).min() > 0.05
    c = sc.centers[:20]
    r = sides * np.sqrt(3) / 2
    d = np.linalg.norm(c[:, None] - c[None], axis=-1) + np.eye(20) * 1e9
    assert (d - r[:, None] - r[None]).min() > 0.09
    assert np.allclose(sc.meta["areas"][:20], 6 * sides ** 2)
