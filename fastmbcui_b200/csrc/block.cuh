// Block PCG building blocks (FP64): the dense products and the small dense
// factorizations of a block conjugate-gradient step over all right-hand
// sides at once (O'Leary, "The block conjugate gradient algorithm and related
// methods", Linear Algebra Appl. 29 (1980); search blocks kept orthonormal
// and of full rank by a rank-revealing Cholesky QR, after Dubrulle,
// "Retooling the method of block conjugate gradients", ETNA 12 (2001)).
//
// Every array is row-major with an explicit leading dimension; n is the
// number of points (rows), k and m the block widths (<= a few hundred).
// All reductions run in a fixed order, so results do not depend on timing.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mbc {
namespace blk {

constexpr int kTile = 64;         // output tile (64 x 64) of the Gram and update kernels
constexpr int kRowsPer = 512;     // rows per Gram partial
constexpr int kKStep = 32;        // rows (Gram) / inner indices (update) staged per pass
constexpr int kThreads = 256;     // 16 x 16 threads, 4 x 4 outputs each
constexpr int kSmallThreads = 1024;

__host__ __device__ inline int gram_chunks(int n) { return (n + kRowsPer - 1) / kRowsPer; }

// part[chunk][i][j] = sum over the chunk's rows r of A[r, i] B[r, j]
// grid (chunks, tiles of ka, tiles of kb)
__global__ void __launch_bounds__(kThreads) gram_partial_kernel(int n, const double *__restrict__ A, int lda,
                                                                 int ka, const double *__restrict__ B, int ldb,
                                                                 int kb, double *__restrict__ part)
{
  __shared__ double sA[kKStep][kTile];
  __shared__ double sB[kKStep][kTile];
  const int chunk = blockIdx.x, ti = blockIdx.y * kTile, tj = blockIdx.z * kTile;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int r0 = chunk * kRowsPer, r1 = min(n, r0 + kRowsPer);
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  for (int rb = r0; rb < r1; rb += kKStep) {
    for (int e = threadIdx.x; e < kKStep * kTile; e += kThreads) {
      const int rr = e / kTile, c = e - rr * kTile, r = rb + rr;
      sA[rr][c] = (r < r1 && ti + c < ka) ? A[(size_t)r * lda + ti + c] : 0.0;
      sB[rr][c] = (r < r1 && tj + c < kb) ? B[(size_t)r * ldb + tj + c] : 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int rr = 0; rr < kKStep; ++rr) {
      double av[4], bv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) av[a] = sA[rr][ty * 4 + a];
#pragma unroll
      for (int b = 0; b < 4; ++b) bv[b] = sB[rr][tx * 4 + b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int i = ti + ty * 4 + a;
    if (i >= ka) continue;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int j = tj + tx * 4 + b;
      if (j < kb) part[((size_t)chunk * ka + i) * kb + j] = acc[a][b];
    }
  }
}

// C[i * ldc + j] = sum over chunks (in order) of part[chunk][i][j]
__global__ void gram_reduce_kernel(int chunks, int ka, int kb, const double *__restrict__ part,
                                   double *__restrict__ C, int ldc)
{
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)ka * kb) return;
  const int i = (int)(t / kb), j = (int)(t - (int64_t)i * kb);
  double s = 0.0;
  for (int c = 0; c < chunks; ++c) s += part[((size_t)c * ka + i) * kb + j];
  C[(size_t)i * ldc + j] = s;
}

// out[r, c] = base[r, c] + sgn * sum_j P[r, j] M[j, c]   (n x m = (n x k)(k x m));
// base may be out (in place) or NULL (zero); nothing is written when *skip
// is set (a failed factorization upstream).  grid (row tiles, column tiles)
__global__ void __launch_bounds__(kThreads) block_update_kernel(int n, int k, int m, const double *__restrict__ P,
                                                                 int ldp, const double *__restrict__ M, int ldm,
                                                                 const double *base, int ldb, double sgn,
                                                                 double *out, int ldo, const int32_t *skip)
{
  if (skip && *skip) return;
  __shared__ double sP[kTile][kKStep + 1];
  __shared__ double sM[kKStep][kTile];
  const int r0 = blockIdx.x * kTile, c0 = blockIdx.y * kTile;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  for (int j0 = 0; j0 < k; j0 += kKStep) {
    for (int e = threadIdx.x; e < kTile * kKStep; e += kThreads) {
      const int rr = e / kKStep, jj = e - rr * kKStep;
      const int r = r0 + rr, j = j0 + jj;
      sP[rr][jj] = (r < n && j < k) ? P[(size_t)r * ldp + j] : 0.0;
    }
    for (int e = threadIdx.x; e < kKStep * kTile; e += kThreads) {
      const int jj = e / kTile, cc = e - jj * kTile;
      const int j = j0 + jj, c = c0 + cc;
      sM[jj][cc] = (j < k && c < m) ? M[(size_t)j * ldm + c] : 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int jj = 0; jj < kKStep; ++jj) {
      double pv[4], mv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) pv[a] = sP[ty * 4 + a][jj];
#pragma unroll
      for (int b = 0; b < 4; ++b) mv[b] = sM[jj][tx * 4 + b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = fma(pv[a], mv[b], acc[a][b]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int r = r0 + ty * 4 + a;
    if (r >= n) continue;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int c = c0 + tx * 4 + b;
      if (c >= m) continue;
      const double v = sgn * acc[a][b];
      out[(size_t)r * ldo + c] = base ? base[(size_t)r * ldb + c] + v : v;
    }
  }
}

// ---------------------------------------------------------------------------
// Small dense kernels.  The k x k matrices are symmetric (Gram matrices) or
// lower triangular (their Cholesky factors), so only the lower triangle is
// read or written.  With `packed` the lower triangle is staged in shared
// memory in packed row order (row i at i (i + 1) / 2), which holds k up to
// kPackedDim; above that the kernels work on the global copy (L1 / L2).  The
// arithmetic and its order are the same either way.
constexpr int kPackedDim = 208;  // 208 * 209 / 2 doubles = 169.8 KB
constexpr int kSolveWarps = 8;   // columns (one warp each) per block of the column-parallel solves

__host__ __device__ constexpr size_t packed_len(int k) { return (size_t)k * (k + 1) / 2; }

// lower-triangle element (i, l), i >= l, of a packed or a row-major matrix
struct Lower {
  double *p;
  int ld;
  int packed;
  __device__ __forceinline__ double &operator()(int i, int l) const
  {
    return packed ? p[(size_t)i * (i + 1) / 2 + l] : p[(size_t)i * ld + l];
  }
};

// lower triangle of src (k x k, ld) -> packed dst; every thread of the block
// takes part and the block is synchronised afterwards
__device__ __forceinline__ void stage_lower(int k, const double *src, int ld, double *dst)
{
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int i = threadIdx.x >> 5; i < k; i += nw)
    for (int l = lane; l <= i; l += 32) dst[(size_t)i * (i + 1) / 2 + l] = src[(size_t)i * ld + l];
  __syncthreads();
}

// In place lower Cholesky of the k x k SPD matrix G (row-major, ld; lower
// triangle read): G = L L^T, L written to the lower triangle (the strict
// upper triangle is left as is).  *flag = 1 on a pivot that is not positive
// (or NaN).  One block of kSmallThreads; with packed, k (k + 1) / 2 doubles
// of dynamic shared memory.
__global__ void __launch_bounds__(kSmallThreads) chol_kernel(int k, double *Gg, int ldg, int32_t *flag, int packed)
{
  extern __shared__ double sm[];
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  if (packed) stage_lower(k, Gg, ldg, sm);
  const Lower G{packed ? sm : Gg, ldg, packed};
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  for (int j = 0; j < k; ++j) {
    if (threadIdx.x == 0) {
      const double d = G(j, j);
      if (!(d > 0.0)) bad = 1;
      G(j, j) = d > 0.0 ? sqrt(d) : 1.0;
    }
    __syncthreads();
    if (bad) break;
    const double djj = G(j, j);
    for (int i = j + 1 + threadIdx.x; i < k; i += blockDim.x) G(i, j) /= djj;
    __syncthreads();
    // trailing update of the lower triangle, one warp per row
    for (int i = j + 1 + warp; i < k; i += nw) {
      const double gij = G(i, j);
      for (int l = j + 1 + lane; l <= i; l += 32) G(i, l) -= gij * G(l, j);
    }
    __syncthreads();
  }
  if (packed) {
    for (int i = warp; i < k; i += nw)
      for (int l = lane; l <= i; l += 32) Gg[(size_t)i * ldg + l] = G(i, l);
  }
  if (threadIdx.x == 0 && bad && flag) *flag = 1;
}

// B (k x m, ldb) <- sgn * (L L^T)^{-1} B for the lower factor L of
// chol_kernel (lower triangle of Lg, ldg).  One warp per column of B,
// kSolveWarps columns per block, grid cdiv(m, kSolveWarps): forward then
// backward substitution in the column-oriented order, the column held in
// shared memory.  Dynamic shared memory: kSolveWarps * k doubles, plus
// packed_len(k) with packed (L staged).  Nothing is done when *skip is set
// (the factorization failed).
__global__ void __launch_bounds__(kSolveWarps * 32) chol_solve_kernel(int k, const double *Lg, int ldg, int m,
                                                                      double *B, int ldb, double sgn,
                                                                      const int32_t *skip, int packed)
{
  extern __shared__ double sm[];
  if (skip && *skip) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double *Lp = sm + (size_t)kSolveWarps * k;
  if (packed) stage_lower(k, Lg, ldg, Lp);
  const Lower L{packed ? Lp : const_cast<double *>(Lg), ldg, packed};
  const int c = blockIdx.x * kSolveWarps + warp;
  if (c >= m) return;
  double *x = sm + (size_t)warp * k;
  for (int i = lane; i < k; i += 32) x[i] = B[(size_t)i * ldb + c];
  __syncwarp();
  // forward: L y = b.  Every lane reads x[j] before the __syncwarp; lane 0
  // stores y_j after it (x[j] is read again only in the backward pass).
  for (int j = 0; j < k; ++j) {
    const double yj = x[j] / L(j, j);
    for (int i = j + 1 + lane; i < k; i += 32) x[i] -= L(i, j) * yj;
    __syncwarp();
    if (lane == 0) x[j] = yj;
  }
  __syncwarp();
  // backward: L^T x = y
  for (int j = k - 1; j >= 0; --j) {
    const double xj = x[j] / L(j, j);
    for (int i = lane; i < j; i += 32) x[i] -= L(j, i) * xj;
    __syncwarp();
    if (lane == 0) x[j] = xj;
  }
  __syncwarp();
  for (int i = lane; i < k; i += 32) B[(size_t)i * ldb + c] = sgn * x[i];
}

constexpr int kOrthMax = 512;  // widest block orth_factor_kernel takes

// Rank-revealing Cholesky of the m x m Gram matrix W (row-major, ld; lower
// triangle read, overwritten by the factor) of a block V (m <= kOrthMax).
// The columns are first scaled to unit norm (the span does not change, and
// a column with a small norm is not mistaken for a dependent one); then,
// with diagonal pivoting, the factorization stops at the first pivot below
// drop^2 times the largest scaled diagonal (or, with drop = 0, not above
// zero).  Writes the factor L of the kept pivots (Pi^T D W D Pi = L L^T on
// them) to W's lower triangle in pivoted order, the pivots perm[m], the
// column scaling scale[m] (D) and *rank = r; orth_t_kernel then forms
// T = D Pi L^{-T}, with V T[:, :r] orthonormal in exact arithmetic.  One
// block of kSmallThreads; with packed, packed_len(m) doubles of dynamic
// shared memory.
__global__ void __launch_bounds__(kSmallThreads) orth_factor_kernel(int m, double *Wg, int ldg, double drop,
                                                                    double *scale, int32_t *perm, int32_t *rank,
                                                                    int packed)
{
  extern __shared__ double sm[];
  __shared__ double s_val[32];
  __shared__ int s_idx[32];
  __shared__ int s_r;
  __shared__ double s_dmax;
  __shared__ double s_scale[kOrthMax];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const Lower W{packed ? sm : Wg, ldg, packed};
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    perm[i] = i;
    const double d = Wg[(size_t)i * ldg + i];
    s_scale[i] = d > 0.0 ? 1.0 / sqrt(d) : 0.0;
  }
  __syncthreads();
  // scaled lower triangle (staged when packed)
  for (int i = warp; i < m; i += nw)
    for (int l = lane; l <= i; l += 32) W(i, l) = Wg[(size_t)i * ldg + l] * (s_scale[i] * s_scale[l]);
  __syncthreads();
  // largest initial diagonal
  {
    double mx = 0.0;
    for (int i = threadIdx.x; i < m; i += blockDim.x) mx = fmax(mx, W(i, i));
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) s_val[warp] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
      double v = 0.0;
      for (int w = 0; w < nw; ++w) v = fmax(v, s_val[w]);
      s_dmax = v;
      s_r = m;
    }
    __syncthreads();
  }
  const double thr = drop > 0.0 ? drop * drop * s_dmax : 0.0;
  // pivoted Cholesky of the symmetric matrix on its lower triangle, rows and
  // columns swapped in place
  for (int j = 0; j < m; ++j) {
    // pivot: the largest remaining diagonal (lowest index on ties)
    double best = -1.0;
    int bi = j;
    for (int i = j + threadIdx.x; i < m; i += blockDim.x) {
      const double d = W(i, i);
      if (d > best) {
        best = d;
        bi = i;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    if (lane == 0) {
      s_val[warp] = best;
      s_idx[warp] = bi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double b = -1.0;
      int p = j;
      for (int w = 0; w < nw; ++w)
        if (s_val[w] > b || (s_val[w] == b && s_idx[w] < p)) {
          b = s_val[w];
          p = s_idx[w];
        }
      s_idx[0] = p;
      s_val[0] = b;
      if (!(b > thr)) s_r = j;
    }
    __syncthreads();
    if (s_r == j) break;
    const int p = s_idx[0];
    if (p != j) {
      // swap rows and columns j < p of the symmetric matrix, on the lower
      // triangle: each x other than j and p pairs two entries; (p, j) stays
      for (int x = threadIdx.x; x < m; x += blockDim.x) {
        if (x == p) continue;
        double *e1, *e2;
        if (x == j) {
          e1 = &W(j, j);
          e2 = &W(p, p);
        } else if (x < j) {
          e1 = &W(j, x);
          e2 = &W(p, x);
        } else if (x < p) {
          e1 = &W(x, j);
          e2 = &W(p, x);
        } else {
          e1 = &W(x, j);
          e2 = &W(x, p);
        }
        const double t = *e1;
        *e1 = *e2;
        *e2 = t;
      }
      if (threadIdx.x == 0) {
        const int32_t q = perm[j];
        perm[j] = perm[p];
        perm[p] = q;
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) W(j, j) = sqrt(W(j, j));
    __syncthreads();
    const double djj = W(j, j);
    for (int i = j + 1 + threadIdx.x; i < m; i += blockDim.x) W(i, j) /= djj;
    __syncthreads();
    // trailing update of the lower triangle, one warp per row
    for (int i = j + 1 + warp; i < m; i += nw) {
      const double wij = W(i, j);
      for (int l = j + 1 + lane; l <= i; l += 32) W(i, l) -= wij * W(l, j);
    }
    __syncthreads();
  }
  const int r = s_r;
  if (packed)
    for (int i = warp; i < r; i += nw)
      for (int l = lane; l <= i; l += 32) Wg[(size_t)i * ldg + l] = W(i, l);
  for (int i = threadIdx.x; i < m; i += blockDim.x) scale[i] = s_scale[i];
  if (threadIdx.x == 0) *rank = r;
}

// T (m x m, ldt; columns c < r written) = D Pi L^{-T} from orth_factor_kernel:
// column c solves L^T x = e_c (x[i] = 0 for i > c) by backward substitution,
// then T[perm[i], c] = x[i] scale[perm[i]].  One warp per column,
// kSolveWarps columns per block, grid cdiv(m, kSolveWarps); dynamic shared
// memory as chol_solve_kernel's (k = m).
__global__ void __launch_bounds__(kSolveWarps * 32) orth_t_kernel(int m, const double *Wg, int ldg,
                                                                  const double *__restrict__ scale,
                                                                  const int32_t *__restrict__ perm,
                                                                  const int32_t *rank, double *T, int ldt, int packed)
{
  extern __shared__ double sm[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r = *rank;
  if (blockIdx.x * kSolveWarps >= r) return;
  double *Lp = sm + (size_t)kSolveWarps * m;
  if (packed) stage_lower(r, Wg, ldg, Lp);
  const Lower L{packed ? Lp : const_cast<double *>(Wg), ldg, packed};
  const int c = blockIdx.x * kSolveWarps + warp;
  if (c >= r) return;
  double *x = sm + (size_t)warp * m;
  for (int i = lane; i < m; i += 32) x[i] = i == c ? 1.0 : 0.0;
  __syncwarp();
  for (int j = c; j >= 0; --j) {
    const double xj = x[j] / L(j, j);
    for (int i = lane; i < j; i += 32) x[i] -= L(j, i) * xj;
    __syncwarp();
    if (lane == 0) x[j] = xj;
  }
  __syncwarp();
  for (int i = lane; i < m; i += 32) {
    const int pi = perm[i];
    T[(size_t)pi * ldt + c] = x[i] * scale[pi];
  }
}

}  // namespace blk
}  // namespace mbc
