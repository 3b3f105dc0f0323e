"""Factor tile shapes (mbc_factor_tiles) and the autotuner on the GPU.

The tile shapes only change how the Gram sums of the supernodal factor are
split over threads and panel passes, so every valid shape must give the same
factor to rounding: FP64 solvers within 1e-8 and FP32 solvers within 1e-3
(norm-wise relative over the factor values: the Gram sums run over 6000
rows, and the supernodal Cholesky amplifies their rounding by the conditioning
of Theta_s: measured in FP64 1.3e-10, and 1.1e-9 with every supernode above
32 rows in the global-memory class).  Invalid shapes are refused; the tuner leaves a valid, faster-or-equal
shape set and the solver factored.
"""
import numpy as np
import pytest

import fastmbcui_b200 as F
from fastmbcui_b200 import scenes as S

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _solver(sc, prec):
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float32, device="cuda")
    plan = F.Plan(sc.y, sc.rho, sc.lam, sc.max_super)
    return F.Solver(plan, x=t(sc.x), nx=t(sc.nx), y=t(sc.y), coef=sc.coef, precision=prec)


@pytest.fixture(scope="module")
def scene():
    return S.ellipsoids_scene(3, 2000, seed=9)


@pytest.mark.parametrize("prec,tol", [(F.MBC_F64, 1e-8), (F.MBC_F32, 1e-3)])
def test_shapes_give_the_same_factor(scene, prec, tol):
    s = _solver(scene, prec)
    ref, _ = s.set_factor_tiles(dict(s.factor_tiles(), tc_min_ns=0)).factor().get_factor()
    for tiles in ({"max_ns": [24, 64, 128], "tile_rows": [16, 16, 16, 16], "tc_min_ns": 0},
                  {"max_ns": [48, 96, 144], "tile_rows": [128, 8, 64, 32], "tc_min_ns": 0},
                  {"max_ns": [8, 16, 32], "tile_rows": [1, 3, 5, 7], "tc_min_ns": 0}):
        got, _ = s.set_factor_tiles(tiles).factor().get_factor()
        assert s.factor_tiles() == tiles
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= tol, tiles


def test_invalid_shapes_are_refused(scene):
    s = _solver(scene, F.MBC_F32)
    for bad in ({"max_ns": [64, 32, 128], "tile_rows": [8, 8, 8, 8]},
                {"max_ns": [32, 64, 200], "tile_rows": [8, 8, 8, 8]},
                {"max_ns": [32, 64, 128], "tile_rows": [0, 8, 8, 8]},
                {"max_ns": [32, 64, 128], "tile_rows": [8, 8, 8, 8], "tc_min_ns": 16},
                {"max_ns": [32, 64, 128], "tile_rows": [8, 8, 8, 8], "tc_min_ns": 200}):
        with pytest.raises(F.MbcError):
            s.set_factor_tiles(bad)


def test_tuner_picks_a_valid_shape(scene):
    s = _solver(scene, F.MBC_F32)
    tiles, ms = s.tune_factor(1)
    assert tiles == s.factor_tiles() and ms > 0
    assert tiles["max_ns"][0] < tiles["max_ns"][1] < tiles["max_ns"][2] <= 144
    Fd = torch.as_tensor(scene.rhs(), dtype=torch.float64, device="cuda")
    _, st = s.solve(Fd, out_dtype=torch.float64, tol=1e-8, max_iters=4000, fp64_recursion=1,
                    true_residual=1)
    assert st["true_relres_max"] <= 1.05e-8
