"""mbc_spatial_order (the reduction order of the INT8 matvec's planes)
against a numpy restatement of the same Morton code (21 bits per axis over
the points' bounding cube, x in the highest of each three bits, ties by
index), and the error bound it lowers."""
import numpy as np
import pytest

import fastmbcui_b200 as F
from fastmbcui_b200 import scenes as S


def morton_np(p):
    p = np.asarray(p, np.float32).astype(np.float64)
    lo = p.min(axis=0)
    ext = (p.max(axis=0) - lo).max()
    scale = ((1 << 21) - 1) / ext if ext > 0 else 0.0
    q = np.clip(np.floor((p - lo) * scale), 0, (1 << 21) - 1).astype(np.uint64)
    code = np.zeros(len(p), np.uint64)
    for b in range(21):
        for d in range(3):
            code |= ((q[:, d] >> np.uint64(b)) & np.uint64(1)) << np.uint64(3 * b + 2 - d)
    return np.lexsort((np.arange(len(p)), code)).astype(np.int32)


@pytest.mark.parametrize("seed", range(3))
def test_matches_numpy_restatement(seed):
    rng = np.random.default_rng(seed)
    p = rng.standard_normal((5000, 3)).astype(np.float32)
    p[:100] = p[100:200]  # exact duplicates: ties by index
    assert np.array_equal(F.spatial_order(p), morton_np(p))


def test_morton_chunks_lower_the_int8_error_bound():
    """The INT8 matvec's per-row error bound sum_c kc max|G_c| (2048-wide
    chunks of the reduction axis): on the 32-ellipsoid trajectory scene,
    walking the sources in Morton order instead of the plan's maximin order
    lowers it about threefold (the far chunks no longer hold near-field
    entries)."""
    base, q, _ = S.trajectory_scene(32, 2000, seed=4, steps=500)
    sc = S.moved(base, q[0])
    plan = F.Plan(sc.y, sc.rho, sc.lam, sc.max_super)
    P, _ = plan.order()
    pinv = np.argsort(P)
    rows = np.random.default_rng(0).choice(sc.nf, 100, replace=False)
    x, nx = sc.x[rows].astype(np.float64), sc.nx[rows].astype(np.float64)

    def bound(order):
        d = x[:, None, :] - sc.y[order][None].astype(np.float64)
        r2 = (d * d).sum(-1)
        g = np.abs((d * nx[:, None, :]).sum(-1)) / (np.sqrt(r2) * r2)
        return sum(g[:, k:k + 2048].max(axis=1) * g[:, k:k + 2048].shape[1] for k in range(0, len(order), 2048))

    plan_b = bound(pinv)
    morton_b = bound(pinv[F.spatial_order(sc.y[pinv])])
    assert np.median(morton_b / plan_b) < 0.5, np.median(morton_b / plan_b)


def test_edge_cases():
    assert F.spatial_order(np.zeros((0, 3))).shape == (0,)
    assert list(F.spatial_order(np.ones((4, 3)))) == [0, 1, 2, 3]
    with pytest.raises(F.MbcError):
        F.spatial_order(np.array([[0.0, np.nan, 0.0]]))
