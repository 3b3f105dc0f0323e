"""mbc_spatial_order (the reduction order of the INT8 matvec's planes)
against a numpy restatement of the same Morton code: 21 bits per axis over
the points' bounding cube, x in the highest of each three bits, ties by
index."""
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


def test_chunks_are_compact():
    """On the 32-ellipsoid scene, in plan (maximin) order every 2048-wide chunk
    spans the scene; in Morton order a chunk covers a small region."""
    sc = S.ellipsoids_scene(32, 2000, seed=4)
    plan = F.Plan(sc.y, sc.rho, sc.lam, sc.max_super)
    P, _ = plan.order()
    yp = sc.y[np.argsort(P)]
    ym = yp[F.spatial_order(yp)]
    ext = lambda a: np.mean([np.ptp(a[k:k + 2048], axis=0).max() for k in range(0, len(a), 2048)])
    assert ext(ym) < 0.25 * ext(yp), (ext(ym), ext(yp))


def test_edge_cases():
    assert F.spatial_order(np.zeros((0, 3))).shape == (0,)
    assert list(F.spatial_order(np.ones((4, 3)))) == [0, 1, 2, 3]
    with pytest.raises(F.MbcError):
        F.spatial_order(np.array([[0.0, np.nan, 0.0]]))
