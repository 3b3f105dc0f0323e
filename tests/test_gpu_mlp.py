"""The warm-start MLP's GPU kernels against the FP64 numpy checker.

Tolerances: forward 1e-5 and gradient 1e-4 relative (norm-wise) -- the
kernels multiply BF16 weights with FP32 activations and accumulate in FP32,
the checker uses the same BF16 weights in FP64.
"""
import numpy as np
import pytest

import mlp_ref as M
from fastmbcui_b200.warmstart import Mlp

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def data():
    rng = np.random.default_rng(1)
    X = rng.standard_normal((300, 40)).astype(np.float32)
    A = rng.standard_normal((40, 12)) / np.sqrt(40)
    T = np.tanh(X @ A).astype(np.float32) + 0.1 * np.sin(3 * X[:, :12]).astype(np.float32)
    return X, T


def test_forward_and_gradient_match_oracle(data):
    X, T = data
    net = Mlp(40, 12, hidden=96, layers=3, seed=3)
    p = net.params()
    Xd, Td = torch.as_tensor(X, device="cuda"), torch.as_tensor(T, device="cuda")
    Y = net.forward(Xd).double().cpu().numpy()
    Yo = M.forward(p, net.dims, X)[-1]
    assert rel(Y, Yo) < 1e-5
    loss, g = net.train_step(Xd, Td, lr=0.0, grads=True)
    lo, go = M.loss_and_grad(p, net.dims, X, T)
    assert abs(loss - lo) < 1e-5 * lo
    assert rel(g.astype(np.float64), go) < 1e-4
    # lr = 0 leaves the parameters as they were
    assert np.array_equal(net.params(), p)


def test_training_reduces_loss_and_is_deterministic(data):
    X, T = data
    Xd, Td = torch.as_tensor(X, device="cuda"), torch.as_tensor(T, device="cuda")
    runs = []
    for _ in range(2):
        net = Mlp(40, 12, hidden=128, layers=3, seed=5)
        first = net.train_step(Xd, Td, lr=0.0)
        for _ in range(300):
            last = net.train_step(Xd, Td, lr=2e-3)
        runs.append((first, last, net.params()))
    (f0, l0, p0), (f1, l1, p1) = runs
    assert l0 < 0.05 * f0, (f0, l0)
    assert np.array_equal(p0, p1) and f0 == f1 and l0 == l1


def test_set_params_roundtrip():
    net = Mlp(7, 3, hidden=16, layers=2, seed=0)
    p = np.random.default_rng(2).standard_normal(net.n_params).astype(np.float32)
    net.set_params(p)
    assert np.array_equal(net.params(), p)
