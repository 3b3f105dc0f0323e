"""The INT8 digit-sliced FP64 matvec, on the CPU.

orc_oz_apply (oracle/mbc_oracle.c) restates, operation for operation, what the
library's INT8 tensor-core kernels compute (matvec_oz.cuh).  Here it is pinned
against an independent numpy mirror of the same specification (bit-exact),
checked against the FP64 product on an MFS operator (relative error bound
written in the test), against the integer-range bound of the level sums, on
non-finite inputs, and in a PCG solve whose residuals are recomputed with the
same operator (the FP64 true residual reaches the tolerance)."""
import numpy as np
import pytest

import oracle as O
from fastmbcui_b200 import scenes as S

W, CHUNK, SHIFT, NONFINITE = 38, 2048, 44, 4096
BIAS = 0x8080808080


def _pow2(e):
    e = np.asarray(e, np.int64)
    out = np.ldexp(1.0, np.clip(e, -1022, 1023).astype(np.int32))
    out = np.where(e < -1022, 0.0, out)
    return np.where(e > 1023, np.inf, out)


def _ceil_exp2(m):
    f, e = np.frexp(m)
    a = np.where(f == 0.5, e - 1, e).astype(np.int64)
    return np.where(m > 0, a, 0)


def _digits(A, a):
    """A (rows x C) with per-row exponents a -> (5, rows, C) int64 digits."""
    with np.errstate(invalid="ignore"):
        T = np.rint((A * _pow2(-a)[:, None]) * 2.0 ** W).astype(np.int64)
    tb = ((T.astype(np.uint64) + np.uint64(BIAS)) ^ np.uint64(BIAS)).astype(np.uint64)
    d = np.empty((5,) + A.shape, np.int64)
    for p in range(5):
        u = ((tb >> np.uint64(8 * (4 - p))) & np.uint64(0xFF)).astype(np.int64)
        d[p] = np.where(u >= 128, u - 256, u)
    return d


def mirror(G, V, coef=1.0):
    """numpy restatement of the same specification (finite inputs)."""
    M, K = G.shape
    R = V.shape[1]
    s = np.zeros((M, R))
    for k0 in range(0, K, CHUNK):
        Gc, Vc = G[:, k0:k0 + CHUNK], V[k0:k0 + CHUNK]
        ea = _ceil_exp2(np.abs(Gc).max(axis=1))
        eb = _ceil_exp2(np.abs(Vc).max(axis=0))
        dg, dv = _digits(Gc, ea), _digits(Vc.T, eb)
        acc = [sum(dg[p] @ dv[l - p].T for p in range(l + 1)) for l in range(5)]
        assert max(np.abs(x).max() for x in acc) < 2 ** 31
        comb = acc[0]
        for l in range(1, 5):
            comb = comb * 256 + acc[l]
        s = s + comb.astype(np.float64) * _pow2(ea[:, None] + eb[None, :] - SHIFT)
    return coef * s


@pytest.fixture(scope="module")
def scene():
    sc = S.ellipsoids_scene(2, 1200, seed=7)
    return sc, sc.dense_K()


def test_oracle_matches_numpy_mirror_bitwise(scene):
    sc, K = scene
    rng = np.random.default_rng(0)
    V = rng.standard_normal((K.shape[1], 5)) * np.array([1.0, 1e-3, 1e5, 3.0, 1e-12])
    V[100:300, 2] = 0.0
    a = O.oz_apply(K, V, coef=sc.coef)
    b = mirror(K, V, coef=sc.coef)
    assert np.array_equal(a, b)
    # transposed operator (the columns direction)
    W = rng.standard_normal((K.shape[0], 3))
    assert np.array_equal(O.oz_apply(K.T, W), mirror(np.ascontiguousarray(K.T), W))


def _bound(G, V):
    """Per-element error bound of the scheme: each product term is off by at
    most 2^-38 (rounding of T) + ~2^-36 (dropped levels) of 2^(a+b) <=
    4 max|g| max|v| of its chunk, so |err| <= 2^-33 sum_c kc max|G_c| max|V_c|."""
    bound = np.zeros((G.shape[0], V.shape[1]))
    for k0 in range(0, G.shape[1], CHUNK):
        kc = min(CHUNK, G.shape[1] - k0)
        bound += (np.abs(G[:, k0:k0 + kc]).max(axis=1)[:, None] * np.abs(V[k0:k0 + kc]).max(axis=0)[None, :] * kc)
    return 2.0 ** -33 * bound


def test_accuracy_against_fp64(scene):
    """Frobenius error <= 1e-9 relative on an MFS operator, and every element
    within the scheme's per-element bound."""
    sc, K = scene
    rng = np.random.default_rng(1)
    V = rng.standard_normal((K.shape[1], 8))
    ref = K @ V
    out = O.oz_apply(K, V)
    assert np.linalg.norm(out - ref) / np.linalg.norm(ref) <= 1e-9
    assert np.all(np.abs(out - ref) <= _bound(K, V))


def test_worst_case_digits_stay_in_int32():
    """The largest level sums: |T| <= 2^38 keeps the top digit in [-64, 64],
    and T = -0x80808080 (scale 2^0, set by one unit entry per row and column
    chunk) makes the four lower digits -128.  Level sums then stay far below
    2^31 for full 2048-wide chunks (the oracle raises if one would not)."""
    K = 2 * CHUNK + 5
    v = -0x80808080 * 2.0 ** -W
    G = np.full((3, K), v)
    V = np.full((K, 2), v)
    for k0 in range(0, K, CHUNK):
        G[:, k0] = 1.0
        V[k0, :] = 1.0
    d = _digits(G[:, 1:CHUNK], np.zeros(3, np.int64))
    assert np.all(d[0] == 0) and np.all(d[1:] == -128)
    out = O.oz_apply(G, V)
    assert np.array_equal(out, mirror(G, V))
    # equal entries with maximal lower digits: the truncation errors add up
    # coherently, but stay inside the per-element bound
    assert np.all(np.abs(out - G @ V) <= _bound(G, V))


def test_non_finite_column_stays_non_finite(scene):
    sc, K = scene
    rng = np.random.default_rng(2)
    V = rng.standard_normal((K.shape[1], 3))
    V[17, 1] = np.nan
    out = O.oz_apply(K, V)
    assert np.all(np.isfinite(out[:, [0, 2]]))
    assert not np.any(np.isfinite(out[:, 1]))
    ref = K @ V
    for c in (0, 2):
        assert np.linalg.norm(out[:, c] - ref[:, c]) / np.linalg.norm(ref[:, c]) <= 1e-9


def test_ragged_and_tiny_shapes():
    rng = np.random.default_rng(3)
    for M, K, R in ((1, 1, 1), (3, 129, 2), (130, 2049, 1), (5, 4097, 7)):
        G = rng.standard_normal((M, K))
        V = rng.standard_normal((K, R))
        out = O.oz_apply(G, V)
        assert np.array_equal(out, mirror(G, V))
        assert np.allclose(out, G @ V, rtol=1e-9, atol=1e-9 * np.abs(G).max() * np.abs(V).max() * K)


def test_pcg_with_the_int8_operator_reaches_fp64_tolerance():
    """Normal equations of a small MFS scene: PCG with both matvecs through
    the INT8 operator, converging only on residuals recomputed with it, ends
    at an FP64 true residual <= 1e-8 in at most 10 % more iterations than
    FP64 PCG."""
    sc = S.ellipsoids_scene(1, 1000, seed=9)
    K = sc.dense_K()
    KT = np.ascontiguousarray(K.T)
    pl = O.plan(sc.y, sc.rho, sc.lam, sc.max_super)
    _, lval, _ = O.factor(O.Op(K.shape[0], K.shape[1], M=K), pl)
    prec = lambda r: O.precond(pl, lval, r[pl["Pinv"]])[pl["P"]]
    A64 = lambda v: KT @ (K @ v)
    Aoz = lambda v: O.oz_apply(KT, O.oz_apply(K, v))
    b = KT @ sc.rhs()[:, 3]
    bn = np.linalg.norm(b)

    def pcg(A, tol, maxit, replace):
        x = np.zeros_like(b)
        r = b.copy()
        z = prec(r)
        p = z.copy()
        rz = r @ z
        it = 0
        while it < maxit:
            q = A(p)
            a = rz / (p @ q)
            x += a * p
            r -= a * q
            it += 1
            if np.linalg.norm(r) < tol * bn:
                if not replace:
                    break
                r = b - A(x)  # converge only on a recomputed residual
                if np.linalg.norm(r) < tol * bn:
                    break
            z = prec(r)
            rz1 = r @ z
            p = z + (rz1 / rz) * p
            rz = rz1
        return x, it

    _, it64 = pcg(A64, 1e-8, 3000, False)
    x, it = pcg(Aoz, 1e-8, 3000, True)
    assert np.linalg.norm(b - A64(x)) / bn <= 1e-8
    assert it <= 1.1 * it64 + 2, (it, it64)
