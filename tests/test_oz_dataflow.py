"""Byte-level CPU replay of the INT8 FP64 matvec kernels' data flow
(fastmbcui_b200/csrc/matvec_oz.cuh), checked bit for bit against the
oracle's restatement of the integer pipeline (orc_oz_apply).

The replay follows the kernels line by line:
  * oz_digits_kernel: per (chunk, row tile) block, every (warp, lane, u,
    k-step) unit writes the five digit bytes of 16 consecutive K positions at
    adig_offset(...) + p * kPlaneBytes + sw128_i8(row, c16), exponents at
    aexp_index(...);
  * oz_pack_b_kernel: per (chunk, group) block, the column exponents and
    every (k-step, column, c16) unit's five digit rows p * np + col of the
    stacked B image;
  * oz_mma_kernel: per CTA (row tile, group) and k-step, the A plane tiles and
    the B image are read back the way a K-major 128-byte-swizzled MMA
    descriptor reads them (element (m, k) at sw128_i8(m, k >> 4) + (k & 15)
    from the descriptor's start; the TF32 kernel validated this mapping on
    the device), every MMA piece (plane p, k-substep kk, rows n0 .. n0 + nn)
    accumulates into the emulated tensor memory at column p * np + n0, and at
    each chunk end the accumulator warps' fold (Horner over the level
    columns l * np + col, FP64 fma with 2^(a + b - 44)) runs.
A mismatch means the kernels' index arithmetic and the integer pipeline
disagree: plane order, stacked-row or level-column mapping, scale order.
"""
import numpy as np
import pytest

import oracle as O

KM, KKS, KD, CHUNK_STEPS, NP_MAX = 128, 128, 5, 16, 96
KCHUNK = KKS * CHUNK_STEPS
PLANE = KM * KKS
W, SHIFT, BIAS, NONFINITE = 38, 44, 0x8080808080, 4096


# --- helpers, as in matvec_oz.cuh -------------------------------------------
def groups_for(R):
    return (R + NP_MAX - 1) // NP_MAX


def np_for(R):
    g = groups_for(R)
    return ((R + g - 1) // g + 15) // 16 * 16


def nks_for(K):
    return (K + KKS - 1) // KKS


def nchunks_for(K):
    return (nks_for(K) + CHUNK_STEPS - 1) // CHUNK_STEPS


def row_tiles(M):
    return (M + KM - 1) // KM


def bstage_bytes(np_):
    return KD * np_ * KKS


def sw128_i8(row, c16):
    return (row >> 3) * 1024 + (row & 7) * 128 + (((c16 ^ row) & 7) << 4)


def adig_offset(rt, ks, p, nks):
    return ((rt * nks + ks) * KD + p) * PLANE


def aexp_index(rt, c, row, nch):
    return (rt * nch + c) * KM + row


def bimg_offset(grp, ks, nks, np_):
    return (grp * nks + ks) * bstage_bytes(np_)


def bexp_index(grp, c, col, nch, np_):
    return (grp * nch + c) * np_ + col


def ceil_exp2(m):
    if m == 0.0:
        return 0
    f, e = np.frexp(m)
    return int(e - 1 if f == 0.5 else e)


def pow2(e):
    if e < -1022:
        return 0.0
    if e > 1023:
        return np.inf
    return float(np.ldexp(1.0, e))


def digit_bytes(v, a):
    """the five digit bytes (top digit first) of rint(v 2^-a 2^38)"""
    T = int(np.rint((v * pow2(-a)) * pow2(W)))
    tb = ((T + BIAS) % (1 << 64)) ^ BIAS
    return [(tb >> (8 * (KD - 1 - p))) & 0xFF for p in range(KD)]


# --- the three kernels --------------------------------------------------------
def digits_kernel(G, rt0=0, cnt=None, mode=3, aexp=None, adig=None):
    """oz_digits_kernel for the matrix G (M x K, FP64, finite) over row tiles
    [rt0, rt0 + cnt): mode 1 exponents, 2 digits (exponents read from aexp),
    3 both; the planes go to the launch's own buffer (slab-local tiles)."""
    M, K = G.shape
    nks, nch = nks_for(K), nchunks_for(K)
    cnt = row_tiles(M) if cnt is None else cnt
    if adig is None:
        adig = np.zeros(cnt * nks * KD * PLANE, np.uint8)
    if aexp is None:
        aexp = np.zeros(row_tiles(M) * nch * KM, np.int64)
    for c in range(nch):
        ks0, ks1 = c * CHUNK_STEPS, min(c * CHUNK_STEPS + CHUNK_STEPS, nks)
        kbase = ks0 * KKS
        kcount = min(KCHUNK, K - kbase)
        for rl in range(cnt):
            rt = rt0 + rl
            for warp in range(8):
                for lane in range(32):
                    sub, c16 = lane >> 3, lane & 7
                    for u in range(4):
                        row = 32 * u + 4 * warp + sub
                        gm = rt * KM + row
                        valid = gm < M
                        if mode & 1:
                            mx = np.abs(G[gm, kbase:kbase + kcount]).max() if valid else 0.0
                            ea = ceil_exp2(mx)
                            if c16 == 0:
                                aexp[aexp_index(rt, c, row, nch)] = ea
                        else:
                            ea = int(aexp[aexp_index(rt, c, row, nch)])
                        if not mode & 2:
                            continue
                        for ks in range(ks0, ks1):
                            kk0 = (ks - ks0) * KKS + c16 * 16
                            tile = adig_offset(rl, ks, 0, nks)
                            for e in range(16):
                                k = kk0 + e
                                b = digit_bytes(G[gm, kbase + k], ea) if (valid and k < kcount) else [0] * KD
                                for p in range(KD):
                                    adig[tile + p * PLANE + sw128_i8(row, c16) + e] = b[p]
    return adig, aexp


def pack_kernel(V):
    """oz_pack_b_kernel for the vector block V (K x R)."""
    K, R = V.shape
    np_, groups, nks, nch = np_for(R), groups_for(R), nks_for(K), nchunks_for(K)
    bimg = np.zeros(groups * nks * bstage_bytes(np_), np.uint8)
    bexp = np.zeros(groups * nch * np_, np.int64)
    for c in range(nch):
        ks0, ks1 = c * CHUNK_STEPS, min(c * CHUNK_STEPS + CHUNK_STEPS, nks)
        kbase = ks0 * KKS
        kcount = min(KCHUNK, K - kbase)
        for grp in range(groups):
            s_exp = []
            for col in range(np_):
                gc = grp * np_ + col
                m = np.abs(V[kbase:kbase + kcount, gc]).max() if gc < R else 0.0
                e = ceil_exp2(m) if np.isfinite(m) else NONFINITE
                s_exp.append(e)
                bexp[bexp_index(grp, c, col, nch, np_)] = e
            for t in range((ks1 - ks0) * np_ * 8):
                col, rest = t % np_, t // np_
                c16, ks = rest & 7, ks0 + (rest >> 3)
                gc = grp * np_ + col
                kk0 = (ks - ks0) * KKS + c16 * 16
                img = bimg_offset(grp, ks, nks, np_)
                for e in range(16):
                    k = kk0 + e
                    b = digit_bytes(V[kbase + k, gc], s_exp[col]) if (gc < R and k < kcount) else [0] * KD
                    for p in range(KD):
                        bimg[img + sw128_i8(p * np_ + col, c16) + e] = b[p]
    return bimg, bexp


def read_tile(buf, base, rows):
    """rows x 128 int8 matrix as a K-major 128B-swizzle descriptor reads it"""
    m = np.arange(rows)[:, None]
    k = np.arange(KKS)[None, :]
    idx = base + (m >> 3) * 1024 + (m & 7) * 128 + ((((k >> 4) ^ m) & 7) << 4) + (k & 15)
    return buf[idx].view(np.int8).astype(np.int64)


def mma_kernel(adig, aexp, bimg, bexp, M, K, R, coef, rt0=0, cnt=None, out=None):
    np_, groups, nks, nch = np_for(R), groups_for(R), nks_for(K), nchunks_for(K)
    cnt = row_tiles(M) if cnt is None else cnt
    out = np.zeros((M, R)) if out is None else out
    for blk in range(cnt * groups):
        rl, grp = blk // groups, blk % groups
        rt = rt0 + rl
        tmem = np.zeros((KM, 512), np.int64)
        sums = np.zeros((KM, np_))
        for ks in range(nks):
            kc = ks % CHUNK_STEPS
            B = read_tile(bimg, bimg_offset(grp, ks, nks, np_), KD * np_)
            for p in range(KD):
                A = read_tile(adig, adig_offset(rl, ks, p, nks), KM)
                nt = np_ * (KD - p)
                for kk in range(KKS // 32):
                    acc = not (kc == 0 and p == 0 and kk == 0)
                    for n0 in range(0, nt, 256):
                        nn = min(256, nt - n0)
                        d = A[:, kk * 32:(kk + 1) * 32] @ B[n0:n0 + nn, kk * 32:(kk + 1) * 32].T
                        assert np.abs(d).max(initial=0) < 2 ** 31
                        c0 = p * np_ + n0
                        tmem[:, c0:c0 + nn] = (tmem[:, c0:c0 + nn] if acc else 0) + d
                        assert np.abs(tmem[:, c0:c0 + nn]).max(initial=0) < 2 ** 31
            if kc == CHUNK_STEPS - 1 or ks == nks - 1:
                c = ks // CHUNK_STEPS
                for row in range(KM):
                    ea = aexp[aexp_index(rt, c, row, nch)]
                    for col in range(np_):
                        comb = 0
                        for l in range(KD):
                            comb = comb * 256 + int(tmem[row, l * np_ + col])
                        w = pow2(int(ea) + int(bexp[bexp_index(grp, c, col, nch, np_)]) - SHIFT)
                        sums[row, col] = float(comb) * w + sums[row, col]  # exact product, one rounding
        for row in range(KM):
            gm = rt * KM + row
            if gm >= M:
                continue
            for col in range(np_):
                gc = grp * np_ + col
                if gc < R:
                    out[gm, gc] = coef * sums[row, col]
    return out


@pytest.mark.parametrize("M,K,R", [(130, 2100, 1), (40, 300, 20), (200, 2300, 100)])
def test_kernel_dataflow_equals_oracle(M, K, R):
    rng = np.random.default_rng(M + K + R)
    # an MFS-like dynamic range: entries spanning six decades, some exact zeros
    G = rng.standard_normal((M, K)) * 10.0 ** rng.uniform(-3, 3, (M, 1)) * 10.0 ** rng.uniform(-3, 0, (1, K))
    G[:, 5:9] = 0.0
    V = rng.standard_normal((K, R)) * 10.0 ** rng.uniform(-2, 2, (1, R))
    adig, aexp = digits_kernel(G)
    bimg, bexp = pack_kernel(V)
    out = mma_kernel(adig, aexp, bimg, bexp, M, K, R, coef=-0.25)
    ref = O.oz_apply(G, V, coef=-0.25)
    assert np.array_equal(out, ref)


def test_slab_mode_equals_full_planes():
    """Planes rebuilt per slab of one row tile (exponents computed once, as
    when the planes do not all fit) give the full-plane result bit for bit."""
    M, K, R = 300, 2100, 12
    rng = np.random.default_rng(11)
    G = rng.standard_normal((M, K)) * 10.0 ** rng.uniform(-2, 2, (M, 1))
    V = rng.standard_normal((K, R))
    bimg, bexp = pack_kernel(V)
    _, aexp = digits_kernel(G, mode=1)  # exponents of every row
    per = 1
    slab = np.zeros(per * nks_for(K) * KD * PLANE, np.uint8)
    out = np.zeros((M, R))
    for r0 in range(0, row_tiles(M), per):
        cnt = min(per, row_tiles(M) - r0)
        slab[:] = 0xA5  # stale bytes from the previous slab must all be overwritten
        digits_kernel(G, rt0=r0, cnt=cnt, mode=2, aexp=aexp, adig=slab)
        mma_kernel(slab, aexp, bimg, bexp, M, K, R, -0.25, rt0=r0, cnt=cnt, out=out)
    assert np.array_equal(out, O.oz_apply(G, V, coef=-0.25))
