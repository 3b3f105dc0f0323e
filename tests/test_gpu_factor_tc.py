"""Tensor-core Gram of the FP32 factor (mbc_factor_tiles.tc_min_ns) on the GPU.

Supernodes with tc_min_ns <= n_s <= 192 form Theta_s = K(:, I_s)^T K(:, I_s)
with tcgen05 3xTF32 MMAs (fastmbcui_b200/csrc/factor_tc.cuh) instead of FP32
FMAs on the CUDA cores; the Cholesky and the KL columns are unchanged.  Both
Grams carry FP32-level rounding (3xTF32 products, FP32 chunk sums), so:
  * the factor with the tensor-core Gram equals the CUDA-core one within
    1e-3 norm-wise (the bound the tile shapes are held to, for the same
    reason: Gram rounding amplified by the conditioning of Theta_s), for the
    point kernel (sets up to 162, so both MMA blocks of the kernel run), the
    dense operator and the matrix-free mesh operator;
  * PCG with the FP64 recursion on that factor reaches the FP64 true
    residual 1e-8 in max(3, 5 %) of the iterations of the CUDA-core factor.
"""
import numpy as np
import pytest

import fastmbcui_b200 as F
from fastmbcui_b200 import scenes as S

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _d(a, dt=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _both(s, tc_min):
    """(factor with the CUDA-core Gram, factor with the tensor-core Gram)."""
    base = s.factor_tiles()
    ref, _ = s.set_factor_tiles(dict(base, tc_min_ns=0)).factor().get_factor()
    assert s.tensor_grams() == 0
    got, _ = s.set_factor_tiles(dict(base, tc_min_ns=tc_min)).factor().get_factor()
    return ref, got


@pytest.fixture(scope="module")
def boxes():
    # 3 boxes of 5000 points over a 120 x 80 floor: N = 24600, rho 4, sets up to 162
    return S.large_scene(n_boxes=3, box_pts=5000, floor=(120, 80))


def test_point_kernel_tensor_gram_matches_cuda_cores(boxes):
    sc = boxes
    plan = F.Plan(sc.y, sc.rho, sc.lam, sc.max_super)
    s = F.Solver(plan, x=_d(sc.x), nx=_d(sc.nx), y=_d(sc.y), coef=sc.coef, precision=F.MBC_F32)
    ref, got = _both(s, 64)
    assert s.tensor_grams() >= 500, s.tensor_grams()
    assert _rel(got, ref) <= 1e-3
    # the same solve on either factor
    Fd = _d(sc.rhs(), torch.float64)
    opts = dict(out_dtype=torch.float64, tol=1e-8, max_iters=8000, iters=True, fp64_recursion=1, true_residual=1)
    _, st_t, it_t = s.solve(Fd, **opts)
    s.set_factor_tiles(dict(s.factor_tiles(), tc_min_ns=0)).factor()
    _, st_c, it_c = s.solve(Fd, **opts)
    assert st_t["n_converged"] == Fd.shape[1] and st_t["true_relres_max"] <= 1.05e-8, st_t
    assert it_t.max() <= max(it_c.max() + 3, 1.05 * it_c.max()), (it_t.max(), it_c.max())


def test_dense_operator_tensor_gram_matches_cuda_cores():
    sc = S.ellipsoids_scene(3, 2000, seed=9)
    plan = F.Plan(sc.y, sc.rho, sc.lam, sc.max_super)
    s = F.Solver(plan, M=_d(sc.dense_K().astype(np.float32)), precision=F.MBC_F32)
    ref, got = _both(s, 32)
    assert s.tensor_grams() > 0
    assert _rel(got, ref) <= 1e-3


def test_mesh_operator_tensor_gram_matches_cuda_cores():
    m = S.mesh_scene([(3, (1.0, 0.8, 0.6), (0.1, 0.2, 0.3), (0.0, 0.0, 0.0), 0.1),
                      (3, (0.7, 0.9, 0.5), (0.3, -0.2, 0.1), (2.6, 0.4, -0.2), 0.1)])
    plan = F.Plan(m["S"], 3.0, 1.5, 2048)
    s = F.Solver(plan, mesh=(_d(m["V"]), _d(m["F"], torch.int32), _d(m["S"])), precision=F.MBC_F32)
    ref, got = _both(s, 32)
    assert s.tensor_grams() > 0
    assert _rel(got, ref) <= 1e-3


def test_fp64_factor_keeps_the_cuda_cores():
    sc = S.ellipsoids_scene(3, 2000, seed=9)
    plan = F.Plan(sc.y, sc.rho, sc.lam, sc.max_super)
    s = F.Solver(plan, x=_d(sc.x), nx=_d(sc.nx), y=_d(sc.y), coef=sc.coef, precision=F.MBC_F64)
    s.set_factor_tiles(dict(s.factor_tiles(), tc_min_ns=32)).factor()
    assert s.tensor_grams() == 0
