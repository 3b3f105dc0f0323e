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
// Small dense kernels: one block of kSmallThreads threads.  With use_smem (the
// caller passes k * k doubles of dynamic shared memory, k <= kSmemDim) the
// k x k matrix is staged in shared memory, otherwise it stays in global
// memory (L1 / L2); the arithmetic and its order are the same either way.
constexpr int kSmemDim = 152;  // 152^2 doubles = 180.5 KB

__device__ __forceinline__ void stage_in(int k, const double *src, int ld, double *dst)
{
  for (int64_t t = threadIdx.x; t < (int64_t)k * k; t += blockDim.x) {
    const int i = (int)(t / k), j = (int)(t % k);
    dst[t] = src[(size_t)i * ld + j];
  }
  __syncthreads();
}

// In place lower Cholesky of the k x k SPD matrix G (row-major, ld):
// G = L L^T, L in the lower triangle (the strict upper triangle is left as
// is).  *flag = 1 on a pivot that is not positive (or NaN).
__global__ void __launch_bounds__(kSmallThreads) chol_kernel(int k, double *Gg, int ldg, int32_t *flag,
                                                             int use_smem)
{
  extern __shared__ double sm[];
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  double *G = Gg;
  int ld = ldg;
  if (use_smem) {
    stage_in(k, Gg, ldg, sm);
    G = sm;
    ld = k;
  }
  __syncthreads();
  for (int j = 0; j < k; ++j) {
    if (threadIdx.x == 0) {
      const double d = G[(size_t)j * ld + j];
      if (!(d > 0.0)) bad = 1;
      G[(size_t)j * ld + j] = d > 0.0 ? sqrt(d) : 1.0;
    }
    __syncthreads();
    if (bad) break;
    const double djj = G[(size_t)j * ld + j];
    for (int i = j + 1 + threadIdx.x; i < k; i += blockDim.x) G[(size_t)i * ld + j] /= djj;
    __syncthreads();
    const int w = k - j - 1;
    for (int64_t t = threadIdx.x; t < (int64_t)w * w; t += blockDim.x) {
      const int i = j + 1 + (int)(t / w), l = j + 1 + (int)(t % w);
      if (l <= i) G[(size_t)i * ld + l] -= G[(size_t)i * ld + j] * G[(size_t)l * ld + j];
    }
    __syncthreads();
  }
  if (use_smem)
    for (int64_t t = threadIdx.x; t < (int64_t)k * k; t += blockDim.x) {
      const int i = (int)(t / k), j = (int)(t % k);
      if (j <= i) Gg[(size_t)i * ldg + j] = sm[t];
    }
  if (threadIdx.x == 0 && bad && flag) *flag = 1;
}

// B (k x m, ldb) <- sgn * (L L^T)^{-1} B, L lower from chol_kernel; nothing
// is done when *skip is set (the factorization failed)
__global__ void __launch_bounds__(kSmallThreads) chol_solve_kernel(int k, const double *Lg, int ldg, int m,
                                                                   double *B, int ldb, double sgn,
                                                                   const int32_t *skip, int use_smem)
{
  extern __shared__ double sm[];
  if (skip && *skip) return;
  const double *L = Lg;
  int ld = ldg;
  if (use_smem) {
    stage_in(k, Lg, ldg, sm);
    L = sm;
    ld = k;
  }
  // forward: L y = b
  for (int j = 0; j < k; ++j) {
    const double ljj = L[(size_t)j * ld + j];
    for (int c = threadIdx.x; c < m; c += blockDim.x) B[(size_t)j * ldb + c] /= ljj;
    __syncthreads();
    const int w = k - j - 1;
    for (int64_t t = threadIdx.x; t < (int64_t)w * m; t += blockDim.x) {
      const int i = j + 1 + (int)(t / m), c = (int)(t % m);
      B[(size_t)i * ldb + c] -= L[(size_t)i * ld + j] * B[(size_t)j * ldb + c];
    }
    __syncthreads();
  }
  // backward: L^T x = y
  for (int j = k - 1; j >= 0; --j) {
    const double ljj = L[(size_t)j * ld + j];
    for (int c = threadIdx.x; c < m; c += blockDim.x) B[(size_t)j * ldb + c] /= ljj;
    __syncthreads();
    for (int64_t t = threadIdx.x; t < (int64_t)j * m; t += blockDim.x) {
      const int i = (int)(t / m), c = (int)(t % m);
      B[(size_t)i * ldb + c] -= L[(size_t)j * ld + i] * B[(size_t)j * ldb + c];
    }
    __syncthreads();
  }
  if (sgn != 1.0)
    for (int64_t t = threadIdx.x; t < (int64_t)k * m; t += blockDim.x) {
      const int i = (int)(t / m), c = (int)(t % m);
      B[(size_t)i * ldb + c] *= sgn;
    }
}

constexpr int kOrthMax = 512;  // widest block orth_factor_kernel takes

// Rank-revealing Cholesky of the m x m Gram matrix W (row-major, ld; destroyed)
// of a block V (m <= kOrthMax).  The columns are first scaled to unit norm
// (the span does not change, and a column with a small norm is not mistaken
// for a dependent one); then, with diagonal pivoting, the factorization
// stops at the first pivot below drop^2 times the largest scaled diagonal
// (or, with drop = 0, not above zero).  Writes T (m x m, ldt, its first r
// columns used) such that V T[:, :r] has orthonormal columns in exact
// arithmetic: T = D Pi U^{-1}, D the column scaling, Pi^T D W D Pi = U^T U on
// the kept pivots; and *rank = r.  Work: perm[m] int32.
__global__ void __launch_bounds__(kSmallThreads) orth_factor_kernel(int m, double *Wg, int ldg, double drop,
                                                                    double *T, int ldt, int32_t *perm,
                                                                    int32_t *rank, int use_smem)
{
  extern __shared__ double sm[];
  double *W = Wg;
  int ld = ldg;
  if (use_smem) {
    stage_in(m, Wg, ldg, sm);
    W = sm;
    ld = m;
  }
  __shared__ double s_val[32];
  __shared__ int s_idx[32];
  __shared__ int s_r;
  __shared__ double s_dmax;
  __shared__ double s_scale[kOrthMax];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    perm[i] = i;
    const double d = W[(size_t)i * ld + i];
    s_scale[i] = d > 0.0 ? 1.0 / sqrt(d) : 0.0;
  }
  __syncthreads();
  for (int64_t t = threadIdx.x; t < (int64_t)m * m; t += blockDim.x) {
    const int i = (int)(t / m), l = (int)(t % m);
    W[(size_t)i * ld + l] *= s_scale[i] * s_scale[l];
  }
  __syncthreads();
  // largest initial diagonal
  {
    double mx = 0.0;
    for (int i = threadIdx.x; i < m; i += blockDim.x) mx = fmax(mx, W[(size_t)i * ld + i]);
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) s_val[warp] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
      double v = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v = fmax(v, s_val[w]);
      s_dmax = v;
      s_r = m;
    }
    __syncthreads();
  }
  const double thr = drop > 0.0 ? drop * drop * s_dmax : 0.0;
  // pivoted Cholesky on the symmetric matrix, lower triangle in the permuted
  // positions: W holds the working matrix with rows / columns swapped in place
  for (int j = 0; j < m; ++j) {
    // pivot: the largest remaining diagonal (lowest index on ties)
    double best = -1.0;
    int bi = j;
    for (int i = j + threadIdx.x; i < m; i += blockDim.x) {
      const double d = W[(size_t)i * ld + i];
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
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
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
      // swap rows and columns j and p of the full symmetric matrix
      for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const double a = W[(size_t)j * ld + i];
        W[(size_t)j * ld + i] = W[(size_t)p * ld + i];
        W[(size_t)p * ld + i] = a;
      }
      __syncthreads();
      for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const double a = W[(size_t)i * ld + j];
        W[(size_t)i * ld + j] = W[(size_t)i * ld + p];
        W[(size_t)i * ld + p] = a;
      }
      if (threadIdx.x == 0) {
        const int32_t q = perm[j];
        perm[j] = perm[p];
        perm[p] = q;
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) W[(size_t)j * ld + j] = sqrt(W[(size_t)j * ld + j]);
    __syncthreads();
    const double djj = W[(size_t)j * ld + j];
    for (int i = j + 1 + threadIdx.x; i < m; i += blockDim.x) W[(size_t)i * ld + j] /= djj;
    __syncthreads();
    // trailing update of the full symmetric trailing block (both triangles,
    // so that later row / column swaps stay consistent)
    const int w = m - j - 1;
    for (int64_t t = threadIdx.x; t < (int64_t)w * w; t += blockDim.x) {
      const int i = j + 1 + (int)(t / w), l = j + 1 + (int)(t % w);
      W[(size_t)i * ld + l] -= W[(size_t)i * ld + j] * W[(size_t)l * ld + j];
    }
    __syncthreads();
  }
  const int r = s_r;
  // U = L^T (r x r upper); T = Pi U^{-1}: solve U X = I column by column
  // (X upper), then scatter the rows by the pivots.  X overwrites T's
  // pivoted rows: T[perm[i], c] = X[i, c].
  for (int64_t t = threadIdx.x; t < (int64_t)m * m; t += blockDim.x) {
    const int i = (int)(t / m), c = (int)(t % m);
    T[(size_t)i * ldt + c] = 0.0;
  }
  __syncthreads();
  // X[i, c] for i <= c < r: back substitution U X = I, U[i][l] = L[l][i] = W[l * ld + i]
  for (int c = threadIdx.x; c < r; c += blockDim.x) {
    for (int i = c; i >= 0; --i) {
      double s = (i == c) ? 1.0 : 0.0;
      for (int l = i + 1; l <= c; ++l) s -= W[(size_t)l * ld + i] * T[(size_t)perm[l] * ldt + c];
      T[(size_t)perm[i] * ldt + c] = s / W[(size_t)i * ld + i];
    }
  }
  __syncthreads();
  for (int64_t t = threadIdx.x; t < (int64_t)m * r; t += blockDim.x) {
    const int i = (int)(t / r), c = (int)(t % r);
    T[(size_t)i * ldt + c] *= s_scale[i];
  }
  if (threadIdx.x == 0) *rank = r;
}

}  // namespace blk
}  // namespace mbc
