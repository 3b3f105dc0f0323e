"""Column compaction of the batched PCG, modelled on the CPU with the same
bookkeeping as run_pcg (fastmbcui_b200/csrc/solver.cu): at each check point,
if at most half of the current columns are active and at least 8 have
stopped, save every current column's x and outcome to the caller's arrays
(through the map `cols` from current to caller columns), gather the active
columns' x, r, p and scalars into the other of two buffer sets, compose the
map, continue; save again at the end.

Compaction must change no column's result: each column's recurrence is its
own.  Checked against the uncompacted batched PCG on the normal equations of
a small MFS scene whose columns stop at very different iterations (per-column
tolerances from 1e-2 to 1e-10, as per-column thresholds allow), so that
several compactions happen."""
import numpy as np
import pytest

import oracle as O
from fastmbcui_b200 import scenes as S

ACTIVE, OK, MAXIT = -1, 0, 1


def batched_pcg(A, prec, B, tol, maxit, check_every, compact):
    n, R = B.shape
    # caller's arrays
    X = np.zeros((n, R))
    status = np.full(R, ACTIVE)
    iters = np.zeros(R, int)
    rr_out = np.zeros(R)
    b2 = (B * B).sum(0)
    thr = np.asarray(tol) ** 2 * b2
    # current view
    cols = np.arange(R)
    x, r, p = X.copy(), B.copy(), np.zeros((n, R))
    st, it_c, rz = status.copy(), iters.copy(), np.full(R, np.inf)
    cb2, cthr, crr = b2.copy(), thr.copy(), b2.copy()
    compactions = 0

    def save():
        X[:, cols] = x
        status[cols] = st
        iters[cols] = it_c
        rr_out[cols] = crr

    for it in range(0, maxit, check_every):
        for _ in range(min(check_every, maxit - it)):
            act = st == ACTIVE
            if not act.any():
                break
            z = prec(r)
            rz1 = (r * z).sum(0)
            beta = np.where(act, rz1 / rz, 0.0)
            rz = np.where(act, rz1, rz)
            p = np.where(act, z + beta * p, p)
            q = A(p)
            pq = (p * q).sum(0)
            alpha = np.where(act, rz / pq, 0.0)
            x = x + alpha * p
            r = r - alpha * q
            s = (r * r).sum(0)
            crr = np.where(act, s, crr)
            it_c = it_c + act
            st = np.where(act & (s < cthr), OK, st)
            st = np.where(act & (st == ACTIVE) & (it_c >= maxit), MAXIT, st)
        if not (st == ACTIVE).any():
            break
        if compact and it + check_every < maxit:
            a = np.nonzero(st == ACTIVE)[0]
            cR = len(st)
            if 0 < len(a) and 2 * len(a) <= cR and cR - len(a) >= 8:
                save()
                x, r, p = x[:, a].copy(), r[:, a].copy(), p[:, a].copy()
                st, it_c, rz, cb2, cthr, crr = st[a], it_c[a], rz[a], cb2[a], cthr[a], crr[a]
                cols = cols[a]
                compactions += 1
    save()
    return X, status, iters, rr_out, compactions


@pytest.fixture(scope="module")
def system():
    sc = S.ellipsoids_scene(2, 400, seed=3)
    K = sc.dense_K()
    pl = O.plan(sc.y, sc.rho, sc.lam, sc.max_super)
    _, lval, _ = O.factor(O.Op(K.shape[0], K.shape[1], M=K), pl)

    def prec(rm):
        out = np.empty_like(rm)
        for c in range(rm.shape[1]):
            out[:, c] = O.precond(pl, lval, rm[pl["Pinv"], c])[pl["P"]]
        return out

    A = lambda V: K.T @ (K @ V)
    B = K.T @ np.concatenate([sc.rhs()] * 6, 1)  # 72 columns
    tol = np.repeat(10.0 ** -np.arange(2, 11), 8)
    return A, prec, B, tol


def test_compaction_changes_no_column(system):
    A, prec, B, tol = system
    X0, s0, i0, r0, c0 = batched_pcg(A, prec, B, tol, 600, 1, compact=False)
    X1, s1, i1, r1, c1 = batched_pcg(A, prec, B, tol, 600, 1, compact=True)
    assert c0 == 0 and c1 >= 2, (c1, i0)
    assert np.array_equal(i0, i1) and np.array_equal(s0, s1)
    assert np.allclose(X1, X0, rtol=1e-12, atol=1e-12 * np.abs(X0).max())
    assert np.allclose(r1, r0, rtol=1e-9, atol=0)
    assert np.all(s1 == OK)
