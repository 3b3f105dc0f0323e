"""Flexible CG around an inexact FP32 inner PCG, on CPU tensors: the
outer-loop logic of fastmbcui_b200.flexible with dense stand-ins for the
device operators (FP64 normal equations of a small scene, the oracle's KL
preconditioner, an FP32 operator perturbed by 6e-6 relative, like the
tensor-core matvec's error).

It must reach the FP64 true residual tolerance, with far fewer FP64 operator
applications than plain FP64 PCG needs iterations, where FP32 PCG alone
stalls far above the tolerance."""
import numpy as np
import pytest

import oracle as O
from fastmbcui_b200 import scenes as S
from fastmbcui_b200.flexible import flexible_cg

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def system():
    sc = S.ellipsoids_scene(1, 1500, seed=5)
    K = sc.dense_K()
    rng = np.random.default_rng(0)
    K32 = torch.as_tensor((K * (1 + 6e-6 * rng.standard_normal(K.shape))).astype(np.float32))
    K64 = torch.as_tensor(K)
    pl = O.plan(sc.y, sc.rho, sc.lam, sc.max_super)
    _, lval, _ = O.factor(O.Op(K.shape[0], K.shape[1], M=K), pl)

    def prec(r):  # columns, original order
        out = np.empty_like(r)
        for c in range(r.shape[1]):
            out[:, c] = O.precond(pl, lval, r[pl["Pinv"], c])[pl["P"]]
        return out

    def apply64(v):
        return K64.T @ (K64 @ v)

    def apply32(v):
        return (K32.T @ (K32 @ v.float())).double()

    def pcg(A, b, iters, tol=0.0):
        x = torch.zeros_like(b)
        r = b.clone()
        z = torch.as_tensor(prec(r.numpy()))
        p = z.clone()
        rz = (r * z).sum(0)
        bn = torch.linalg.norm(b, dim=0)
        it = 0
        while it < iters and bool((torch.linalg.norm(r, dim=0) > tol * bn).any()):
            q = A(p)
            a = rz / (p * q).sum(0)
            x = x + a * p
            r = r - a * q
            z = torch.as_tensor(prec(r.numpy()))
            rz1 = (r * z).sum(0)
            p = z + (rz1 / rz) * p
            rz = rz1
            it += 1
        return x, it

    b = K64.T @ torch.as_tensor(sc.rhs()[:, [0, 4]], dtype=torch.float64)
    return apply64, apply32, pcg, b


def test_fp32_pcg_alone_stalls(system):
    apply64, apply32, pcg, b = system
    x, _ = pcg(apply32, b, 600)
    rel = torch.linalg.norm(b - apply64(x), dim=0) / torch.linalg.norm(b, dim=0)
    assert float(rel.max()) > 1e-6


def test_flexible_cg_reaches_fp64_tolerance_with_few_fp64_applies(system):
    apply64, apply32, pcg, b = system
    _, it64 = pcg(apply64, b, 5000, tol=1e-8)

    def inner(r):
        return pcg(apply32, r, 30)[0]

    x, info = flexible_cg(apply64, inner, b, tol=1e-8, keep=20)
    rel = torch.linalg.norm(b - apply64(x), dim=0) / torch.linalg.norm(b, dim=0)
    assert float(rel.max()) <= 1e-8
    assert info["converged"] == b.shape[1]
    assert info["fp64_applies"] * 4 < it64, (info, it64)


def test_frozen_and_zero_columns(system):
    apply64, apply32, pcg, b = system
    b3 = torch.cat([b, torch.zeros_like(b[:, :1])], dim=1)

    def inner(r):
        return pcg(apply32, r, 30)[0]

    x, info = flexible_cg(apply64, inner, b3, tol=1e-8)
    assert torch.isfinite(x).all() and bool((x[:, 2] == 0).all())
    assert info["relres_max"] <= 1e-8


def test_warm_start(system):
    apply64, apply32, pcg, b = system

    def inner(r):
        return pcg(apply32, r, 30)[0]

    x, cold = flexible_cg(apply64, inner, b, tol=1e-8)
    # a start near the solution (as along a trajectory) takes fewer FP64 applications
    x0 = x * (1 + 1e-3 * torch.randn(x.shape, dtype=x.dtype, generator=torch.Generator().manual_seed(0)))
    x1, warm = flexible_cg(apply64, inner, b, tol=1e-8, x0=x0)
    rel = torch.linalg.norm(b - apply64(x1), dim=0) / torch.linalg.norm(b, dim=0)
    assert float(rel.max()) <= 1e-8
    assert warm["fp64_applies"] < cold["fp64_applies"], (warm, cold)
