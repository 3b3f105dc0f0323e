"""The warm-start MLP's CPU checker against finite differences."""
import numpy as np

import mlp_ref as M


def _loss64(p, dims, X, T):
    a = X
    off = 0
    for l in range(len(dims) - 1):
        n, k = dims[l + 1], dims[l]
        W = p[off:off + n * k].reshape(n, k)
        off += n * k
        b = p[off:off + n]
        off += n
        z = a @ W.T + b
        a = z if l == len(dims) - 2 else np.tanh(z)
    return 0.5 * np.sum((a - T) ** 2) / a.size


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    dims = [5, 8, 8, 3]
    n = sum(dims[l + 1] * dims[l] + dims[l + 1] for l in range(3))
    # parameters exactly representable in BF16, so the rounding is the identity
    p = M.bf16_round(rng.standard_normal(n).astype(np.float32) * 0.5).astype(np.float32)
    X, T = rng.standard_normal((7, 5)), rng.standard_normal((7, 3))
    loss, g = M.loss_and_grad(p, dims, X, T)
    pp = p.astype(np.float64)
    assert abs(loss - _loss64(pp, dims, X, T)) < 1e-14
    fd = np.empty(n)
    for i in range(n):
        e = np.zeros(n)
        e[i] = 1e-6
        fd[i] = (_loss64(pp + e, dims, X, T) - _loss64(pp - e, dims, X, T)) / 2e-6
    assert np.abs(fd - g).max() < 1e-8 * np.abs(fd).max() + 1e-12


def test_bf16_rounding():
    a = np.array([1.0, 1.00390625, 1.005859375, -3.3e-5, 65504.0], np.float32)
    r = M.bf16_round(a)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: to even (1.0); 1.0058 rounds up
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125
    assert np.all(np.abs(r - a) <= np.abs(a) * 2.0 ** -8)
