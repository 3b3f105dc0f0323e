"""The warm-start network on libmbc's own kernels (mbc_mlp_*).

``Mlp`` is a small MLP (tanh hidden layers, linear output, BF16 weights in the
products, FP32 accumulation, Adam on FP32 master weights), trained and
evaluated on the GPU.  No counterpart in the reference: its PCG always starts
from zero (src/kl_chol.cu:930-940); here a predicted warm start seeds the
PCG, which still runs to the same FP64 true-residual tolerance.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, load


class Mlp:
    def __init__(self, n_in: int, n_out: int, hidden: int = 256, layers: int = 3, seed: int = 0):
        self.dims = [n_in] + [hidden] * layers + [n_out]
        h = C.c_void_p()
        check(load().mbc_mlp_create(n_in, hidden, layers, n_out, seed, C.byref(h)), "mbc_mlp_create")
        self._h = h
        cnt = C.c_int64()
        check(load().mbc_mlp_num_params(h, C.byref(cnt)), "mbc_mlp_num_params")
        self.n_params = int(cnt.value)

    def __del__(self):
        h = getattr(self, "_h", None)
        L = getattr(_lib, "_lib", None) if _lib is not None else None
        if h and L is not None:
            L.mbc_mlp_destroy(h)
            self._h = None

    @staticmethod
    def _sp():
        import torch

        return C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def params(self) -> np.ndarray:
        p = np.empty(self.n_params, np.float32)
        check(load().mbc_mlp_get_params(self._h, p.ctypes.data), "mbc_mlp_get_params")
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.n_params
        check(load().mbc_mlp_set_params(self._h, p.ctypes.data), "mbc_mlp_set_params")

    def forward(self, X):
        import torch

        X = X.contiguous().float()
        Y = torch.empty((X.shape[0], self.dims[-1]), dtype=torch.float32, device=X.device)
        check(load().mbc_mlp_forward(self._h, X.shape[0], X.data_ptr(), Y.data_ptr(), self._sp()),
              "mbc_mlp_forward")
        return Y

    def train_step(self, X, T, lr: float, grads: bool = False):
        """One Adam step (lr > 0) or a pure gradient evaluation (lr = 0);
        returns the batch loss (and the gradient when asked)."""
        X, T = X.contiguous().float(), T.contiguous().float()
        loss = C.c_double()
        g = np.empty(self.n_params, np.float32) if grads else None
        check(load().mbc_mlp_train_step(self._h, X.shape[0], X.data_ptr(), T.data_ptr(), float(lr),
                                        C.byref(loss), None if g is None else g.ctypes.data, self._sp()),
              "mbc_mlp_train_step")
        return (loss.value, g) if grads else loss.value


# --------------------------------------------------------------------------
# Learned warm start along a rigid-body trajectory.
#
# x0(t) = x(t-1) + U H(t): U (n x 6) holds each body's own rigid-mode
# solution when alone (base pose, on its own sources); for every body b and
# each of its neighbours c (itself and the 8 nearest), the network predicts the
# 6 x 6 block H[c][b] that moves the strengths of body c for the modes of body
# b from the previous step to this one.  Inputs: the pose increments of both
# bodies, their poses and shapes, and their offset.
# --------------------------------------------------------------------------

N_NEIGHBOURS = 8
N_FEATURES = 48


def isolated_basis(sc, tol=1e-10, device="cuda"):
    """U (n x 6, float32, device): for each body alone, its solution for its
    own 6 rigid modes, on its own sources (original order)."""
    import torch

    from . import Plan, Solver
    from . import scenes as S

    U = torch.zeros((sc.n, 6), dtype=torch.float32, device=device)
    rp, sp = sc.body_ptr(), np.searchsorted(sc.src_body, np.arange(sc.n_bodies + 1))
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32), device=device)
    for b in range(sc.n_bodies):
        r0, r1, s0, s1 = rp[b], rp[b + 1], sp[b], sp[b + 1]
        sub = S.Scene(name="body", x=sc.x[r0:r1], nx=sc.nx[r0:r1], y=sc.y[s0:s1],
                      row_body=np.zeros(r1 - r0, np.int32), src_body=np.zeros(s1 - s0, np.int32),
                      centers=sc.centers[b:b + 1], coef=sc.coef, rho=sc.rho, lam=sc.lam, max_super=sc.max_super)
        plan = Plan(sub.y, sub.rho, sub.lam, sub.max_super)
        s = Solver(plan, x=t(sub.x), nx=t(sub.nx), y=t(sub.y), coef=sub.coef, precision=_lib.MBC_F32).factor()
        X, _ = s.solve(t(sub.rhs()), out_dtype=torch.float32, tol=tol, max_iters=4000)
        U[s0:s1] = X
    return U


def neighbour_pairs(centers, k=N_NEIGHBOURS):
    """(c, b) pairs: every body b with itself and its k nearest bodies c."""
    c = np.asarray(centers, np.float64)
    d = np.linalg.norm(c[:, None] - c[None], axis=-1)
    out = []
    for b in range(c.shape[0]):
        order = np.argsort(d[b], kind="stable")[: k + 1]
        out += [(int(cc), b) for cc in order]
    return np.array(out, np.int32)


def pair_features(pairs, q_prev, q_cur, base_centers, axes, base_rot):
    """Network inputs (P x N_FEATURES) of the pairs (c, b) at a step."""
    from .scenes import rotvec_matrix

    q_prev, q_cur = np.asarray(q_prev, np.float64), np.asarray(q_cur, np.float64)
    cen = np.asarray(base_centers, np.float64) + q_cur[:, :3]
    Rw = [rotvec_matrix(q_cur[b, 3:6]) @ base_rot[b] for b in range(q_cur.shape[0])]
    f = np.zeros((len(pairs), N_FEATURES))
    for i, (c, b) in enumerate(pairs):
        dq_b, dq_c = (q_cur[b] - q_prev[b]) * 100.0, (q_cur[c] - q_prev[c]) * 100.0
        d = cen[c] - cen[b]
        r = float(np.linalg.norm(d))
        inv = 1.0 / r if r > 0 else 0.0
        f[i] = np.concatenate([dq_b, dq_c, d * inv, [inv, inv ** 3, 1.0 if c == b else 0.0],
                               Rw[b].ravel(), Rw[c].ravel(), axes[b], axes[c], q_cur[b, 3:6], q_cur[c, 3:6]])
    return f.astype(np.float32)


def pair_targets(U, D, sc, pairs):
    """Least-squares H[c][b] (P x 36) with U[c sources] H = D[c sources, 6b:6b+6]."""
    import torch

    sp = np.searchsorted(sc.src_body, np.arange(sc.n_bodies + 1))
    out = torch.empty((len(pairs), 36), dtype=torch.float64, device=U.device)
    for i, (c, b) in enumerate(pairs):
        Uc = U[sp[c]:sp[c + 1]].double()
        Dc = D[sp[c]:sp[c + 1], 6 * b:6 * b + 6].double()
        out[i] = torch.linalg.lstsq(Uc, Dc).solution.reshape(-1)
    return out.float()


class WarmStart:
    """A trained network with its input / output scalings."""

    def __init__(self, net: Mlp, x_mean, x_std, y_std):
        self.net, self.x_mean, self.x_std, self.y_std = net, x_mean, x_std, float(y_std)

    def predict_H(self, feats):
        import torch

        X = torch.as_tensor((feats - self.x_mean) / self.x_std, dtype=torch.float32, device="cuda")
        return self.net.forward(X) * self.y_std

    def apply(self, X_prev, U, sc_src_body_dev, n_bodies, pairs, feats):
        """x0 = x(t-1) + U H (device, float32, n x R)."""
        import torch

        Hp = self.predict_H(feats)
        H = torch.zeros((n_bodies * n_bodies, 36), dtype=torch.float32, device=X_prev.device)
        idx = torch.as_tensor(pairs[:, 0].astype(np.int64) * n_bodies + pairs[:, 1], device=X_prev.device)
        H[idx] = Hp
        X0 = X_prev.clone().contiguous()
        check(load().mbc_warm_correct(X0.shape[0], X0.shape[1], sc_src_body_dev.data_ptr(), n_bodies,
                                      U.data_ptr(), H.data_ptr(), X0.data_ptr(),
                                      C.c_void_p(torch.cuda.current_stream().cuda_stream)), "mbc_warm_correct")
        return X0

    def save(self, path):
        np.savez_compressed(path, params=self.net.params(), dims=np.array(self.net.dims), x_mean=self.x_mean,
                            x_std=self.x_std, y_std=self.y_std)

    @classmethod
    def load(cls, path):
        z = np.load(path)
        dims = [int(d) for d in z["dims"]]
        net = Mlp(dims[0], dims[-1], hidden=dims[1], layers=len(dims) - 2)
        net.set_params(z["params"])
        return cls(net, z["x_mean"], z["x_std"], float(z["y_std"]))


# --------------------------------------------------------------------------
# Learned cold start: a scene with no history (the first step of a
# trajectory, an independent scene of a batch).  x0 = U H over the pairs
# (c, b): for c = b the block that turns the isolated solution of body b into
# its share of the coupled one, for its neighbours c the response of body c to
# the motion of body b, both predicted from the pair's geometry.
# --------------------------------------------------------------------------

N_COLD_FEATURES = 36


def cold_features(pairs, q_cur, base_centers, axes, base_rot):
    """Network inputs (P x N_COLD_FEATURES) of the pairs (c, b) of one pose."""
    from .scenes import rotvec_matrix

    q_cur = np.asarray(q_cur, np.float64)
    cen = np.asarray(base_centers, np.float64) + q_cur[:, :3]
    Rq = [rotvec_matrix(q_cur[b, 3:6]) for b in range(q_cur.shape[0])]
    Rw = [Rq[b] @ base_rot[b] for b in range(q_cur.shape[0])]
    f = np.zeros((len(pairs), N_COLD_FEATURES))
    for i, (c, b) in enumerate(pairs):
        d = cen[c] - cen[b]
        r = float(np.linalg.norm(d))
        inv = 1.0 / r if r > 0 else 0.0
        f[i] = np.concatenate([d * inv, [inv, inv ** 3, 1.0 if c == b else 0.0], Rw[b].ravel(), Rw[c].ravel(),
                               axes[b], axes[c], q_cur[b, 3:6], q_cur[c, 3:6]])
    return f.astype(np.float32)


def _self_blocks(q_cur, n_bodies):
    """H[b][b] = blockdiag(Rq^T, Rq^T): the isolated solution of body b
    (base pose) expressed in the world modes of its current pose."""
    from .scenes import rotvec_matrix

    H = np.zeros((n_bodies * n_bodies, 36), np.float32)
    for b in range(n_bodies):
        RqT = rotvec_matrix(np.asarray(q_cur[b, 3:6], np.float64)).T
        G = np.zeros((6, 6))
        G[:3, :3] = RqT
        G[3:, 3:] = RqT
        H[b * n_bodies + b] = G.ravel()
    return H


class ColdStart(WarmStart):
    """x0 = U H for a scene without history: the self blocks exact (each
    body's isolated solution at its pose), the neighbour blocks from the
    network.  Measured: network-predicted self blocks, even at 4 % error,
    cost more iterations than x0 = 0, because their error lies along the
    operator's ill-conditioned directions."""

    def start(self, n, R, U, src_body_dev, n_bodies, pairs, feats, q_cur):
        import torch

        H = torch.as_tensor(_self_blocks(q_cur, n_bodies), device=U.device)
        nbr = pairs[:, 0] != pairs[:, 1]
        if nbr.any():
            Hp = self.predict_H(feats[nbr])
            idx = torch.as_tensor(pairs[nbr, 0].astype(np.int64) * n_bodies + pairs[nbr, 1], device=U.device)
            H[idx] = Hp
        X0 = torch.zeros((n, R), dtype=torch.float32, device=U.device)
        check(load().mbc_warm_correct(n, R, src_body_dev.data_ptr(), n_bodies, U.data_ptr(), H.data_ptr(),
                                      X0.data_ptr(), C.c_void_p(torch.cuda.current_stream().cuda_stream)),
              "mbc_warm_correct")
        return X0


def isolated_start(n, R, U, src_body_dev, n_bodies, q_cur):
    """x0 = each body's own isolated solution, rotated to its pose (no network)."""
    import torch

    X0 = torch.zeros((n, R), dtype=torch.float32, device=U.device)
    Hd = torch.as_tensor(_self_blocks(q_cur, n_bodies), device=U.device)
    check(load().mbc_warm_correct(n, R, src_body_dev.data_ptr(), n_bodies, U.data_ptr(), Hd.data_ptr(),
                                  X0.data_ptr(), C.c_void_p(torch.cuda.current_stream().cuda_stream)),
          "mbc_warm_correct")
    return X0
