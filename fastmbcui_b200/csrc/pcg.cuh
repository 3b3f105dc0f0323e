// Batched PCG kernels (kl_chol.cu:891-1088 for one column, here R columns at
// once with per-column alpha, beta and stopping).  Vectors are n x R
// row-major in the new (fine-to-coarse) order, arithmetic type T; every PCG
// scalar and every dot product is FP64 (partial sums per block, then one
// deterministic reduction).  Elementwise kernels use a 2-D block: x over RHS
// columns, y over points.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mbc {

// COL_STAGNANT: replacement mode only -- three consecutive replacements
// found the true residual less than halved: the FP32 recursion has reached
// its attainable accuracy and the column is finished in FP64.
enum ColStatus : int32_t { COL_ACTIVE = -1, COL_OK = 0, COL_MAXIT = 1, COL_BREAKDOWN = 2, COL_STAGNANT = 3 };

struct PcgScalars {
  double *rz, *b2, *thr, *alpha, *beta, *rr, *pt;
  double *rr_ref;  // residual replacement: |r|^2 at the last replacement
  int32_t *stall;  // residual replacement: consecutive replacements without progress
  int32_t *status, *iters;
  int32_t *done;   // 1 when no column is active
  int32_t *want;   // residual replacement requested (set by RED_CHECK)
  int32_t maxit;
  double tol2;
  double drop2;    // > 0: replacement mode, replace once |r|^2 < drop2 * rr_ref
  int32_t stall_check;  // replacement mode: 1 = mark columns stagnant (COL_STAGNANT)
};

// Block reduction over threadIdx.y of one double per thread; thread (x, 0)
// writes the block sum for column x.
__device__ __forceinline__ double block_sum_y(double v, double *red)
{
  const int tx = threadIdx.x, ty = threadIdx.y;
  red[ty * blockDim.x + tx] = v;
  __syncthreads();
  for (int h = blockDim.y / 2; h > 0; h >>= 1) {
    if (ty < h) red[ty * blockDim.x + tx] += red[(ty + h) * blockDim.x + tx];
    __syncthreads();
  }
  return red[tx];
}

// u = L^T r   (u_j = sum over column j of L)
template <typename T, typename LT>
__global__ void precond_lt_kernel(int n, int R, const int32_t *__restrict__ lptr,
                                  const int32_t *__restrict__ lind, const LT *__restrict__ lval,
                                  const T *__restrict__ r, T *__restrict__ u,
                                  const int32_t *__restrict__ done)
{
  if (done && *done) return;
  const int c = blockIdx.y * blockDim.x + threadIdx.x;
  const int j = blockIdx.x * blockDim.y + threadIdx.y;
  if (c >= R || j >= n) return;
  T acc = T(0);
  const int k1 = lptr[j + 1];
  for (int k = lptr[j]; k < k1; ++k) acc = fma((T)lval[k], r[(size_t)lind[k] * R + c], acc);
  u[(size_t)j * R + c] = acc;
}

// z = L u (gather over the row-wise view), fused part = r . z per block
template <typename T, typename LT>
__global__ void precond_l_kernel(int n, int R, const int32_t *__restrict__ rptr,
                                 const int32_t *__restrict__ rcol, const int32_t *__restrict__ rmap,
                                 const LT *__restrict__ lval, const T *__restrict__ u,
                                 T *__restrict__ z, const T *__restrict__ rv,
                                 double *__restrict__ part, const int32_t *__restrict__ done)
{
  if (done && *done) return;
  extern __shared__ double red[];
  const int c = blockIdx.y * blockDim.x + threadIdx.x;
  const int i = blockIdx.x * blockDim.y + threadIdx.y;
  double d = 0.0;
  if (c < R && i < n) {
    T acc = T(0);
    const int t1 = rptr[i + 1];
    for (int t = rptr[i]; t < t1; ++t) acc = fma((T)lval[rmap[t]], u[(size_t)rcol[t] * R + c], acc);
    z[(size_t)i * R + c] = acc;
    d = (double)rv[(size_t)i * R + c] * (double)acc;
  }
  const double s = block_sum_y(d, red);
  if (threadIdx.y == 0 && c < R) part[(size_t)blockIdx.x * R + c] = s;
}

// part = a . b per block (a, b n x R)
template <typename T>
__global__ void dot_partial_kernel(int n, int R, const T *__restrict__ a, const T *__restrict__ b,
                                   double *__restrict__ part)
{
  extern __shared__ double red[];
  const int c = blockIdx.y * blockDim.x + threadIdx.x;
  const int i = blockIdx.x * blockDim.y + threadIdx.y;
  double d = 0.0;
  if (c < R && i < n) d = (double)a[(size_t)i * R + c] * (double)b[(size_t)i * R + c];
  const double s = block_sum_y(d, red);
  if (threadIdx.y == 0 && c < R) part[(size_t)blockIdx.x * R + c] = s;
}

// x += alpha p; r -= alpha t; part = r . r   (x may be FP64 while p, r are T)
template <typename T, typename XT>
__global__ void update_xr_kernel(int n, int R, const double *__restrict__ alpha,
                                 const T *__restrict__ p, const T *__restrict__ t,
                                 XT *__restrict__ x, T *__restrict__ r, double *__restrict__ part,
                                 const int32_t *__restrict__ done)
{
  if (done && *done) return;
  extern __shared__ double red[];
  const int c = blockIdx.y * blockDim.x + threadIdx.x;
  const int i = blockIdx.x * blockDim.y + threadIdx.y;
  double d = 0.0;
  if (c < R && i < n) {
    const size_t o = (size_t)i * R + c;
    const double a = alpha[c];
    const XT xv = (XT)((double)x[o] + a * (double)p[o]);
    const T rv = (T)((double)r[o] - a * (double)t[o]);
    x[o] = xv;
    r[o] = rv;
    d = (double)rv * (double)rv;
  }
  const double s = block_sum_y(d, red);
  if (threadIdx.y == 0 && c < R) part[(size_t)blockIdx.x * R + c] = s;
}

// p = z + beta p (active columns only)
template <typename T>
__global__ void update_p_kernel(int n, int R, const double *__restrict__ beta,
                                const int32_t *__restrict__ status, const T *__restrict__ z,
                                T *__restrict__ p, const int32_t *__restrict__ done)
{
  if (done && *done) return;
  const int c = blockIdx.y * blockDim.x + threadIdx.x;
  const int i = blockIdx.x * blockDim.y + threadIdx.y;
  if (c >= R || i >= n || status[c] != COL_ACTIVE) return;
  const size_t o = (size_t)i * R + c;
  p[o] = (T)((double)z[o] + beta[c] * (double)p[o]);
}

enum ReduceMode : int32_t {
  RED_STORE = 0,   // out[c] = s
  RED_INIT_B = 1,  // b2 = s, thr = tol^2 s, status ACTIVE unless |b|^2 < 1e-16
  RED_ALPHA = 2,   // alpha = rz / s (breakdown if s <= 0 or NaN)
  RED_CHECK = 3,   // rr = s, iters++, converge / max-iteration test, done flag
  RED_BETA = 4,    // beta = s / rz, rz = s
  RED_REPLACE = 5  // true |r|^2 after a residual replacement: rr = rr_ref = s, converge test
};

// One block of 1024 threads: warp per column, lanes over the partial blocks.
__global__ void __launch_bounds__(1024) reduce_kernel(int nblk, int R,
                                                      const double *__restrict__ part,
                                                      int32_t mode, PcgScalars sc,
                                                      double *__restrict__ out)
{
  if (mode != RED_INIT_B && mode != RED_STORE && mode != RED_REPLACE && sc.done && *sc.done) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int any = 0;
  for (int c = warp; c < R; c += 32) {
    double s = 0.0;
    for (int b = lane; b < nblk; b += 32) s += part[(size_t)b * R + c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
      switch (mode) {
        case RED_STORE:
          out[c] = s;
          break;
        case RED_INIT_B:
          sc.b2[c] = s;
          sc.thr[c] = sc.tol2 * s;
          if (sc.rr_ref) sc.rr_ref[c] = s;
          if (sc.stall) sc.stall[c] = 0;
          if (sc.status[c] == COL_ACTIVE && s < 1e-16) {
            sc.status[c] = COL_OK;  // kl_chol.cu:950-953: zero right-hand side
            sc.rr[c] = 0.0;
          }
          break;
        case RED_ALPHA:
          if (sc.status[c] == COL_ACTIVE) {
            sc.pt[c] = s;
            if (!(s > 0.0) || !(sc.rz[c] == sc.rz[c])) {
              sc.status[c] = COL_BREAKDOWN;
              sc.alpha[c] = 0.0;
            } else {
              sc.alpha[c] = sc.rz[c] / s;
            }
          } else {
            sc.alpha[c] = 0.0;
          }
          break;
        case RED_CHECK:
          if (sc.status[c] == COL_ACTIVE) {
            sc.rr[c] = s;
            sc.iters[c] += 1;
            if (!(s == s)) {
              sc.status[c] = COL_BREAKDOWN;
            } else if (sc.drop2 > 0.0) {
              // replacement mode: convergence is only declared on a true
              // FP64 residual, so ask for one
              if (s < sc.thr[c] || s < sc.drop2 * sc.rr_ref[c]) *sc.want = 1;
              if (sc.iters[c] >= sc.maxit) sc.status[c] = COL_MAXIT;
            } else if (s < sc.thr[c]) {
              sc.status[c] = COL_OK;
            } else if (sc.iters[c] >= sc.maxit) {
              sc.status[c] = COL_MAXIT;
            }
          }
          break;
        case RED_REPLACE:
          if (sc.status[c] == COL_ACTIVE || sc.status[c] == COL_MAXIT) {
            const double prev = sc.rr_ref[c];
            sc.rr[c] = s;
            sc.rr_ref[c] = s;
            if (!(s == s)) {
              sc.status[c] = COL_BREAKDOWN;
            } else if (s < sc.thr[c]) {
              sc.status[c] = COL_OK;
            } else if (sc.stall_check) {
              sc.stall[c] = s > 0.25 * prev ? sc.stall[c] + 1 : 0;
              if (sc.stall[c] >= 3 && sc.status[c] == COL_ACTIVE) sc.status[c] = COL_STAGNANT;
            }
          }
          break;
        case RED_BETA:
          if (sc.status[c] == COL_ACTIVE) {
            sc.beta[c] = s / sc.rz[c];
            sc.rz[c] = s;
          } else {
            sc.beta[c] = 0.0;
          }
          break;
      }
      if (sc.status && sc.status[c] == COL_ACTIVE) any = 1;
    }
  }
  if (mode == RED_CHECK || mode == RED_INIT_B || mode == RED_ALPHA || mode == RED_REPLACE) {
    any = __syncthreads_or(any);
    if (threadIdx.x == 0 && sc.done) *sc.done = any ? 0 : 1;
  }
}

// ---- small helpers --------------------------------------------------------

// dst[P[o], c] = (T) src[o, c]  (original order -> new order, type change)
template <typename S, typename D>
__global__ void permute_in_kernel(int n, int R, const int32_t *__restrict__ P,
                                  const S *__restrict__ src, D *__restrict__ dst)
{
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n * R) return;
  const int o = (int)(idx / R), c = (int)(idx - (int64_t)o * R);
  dst[(size_t)P[o] * R + c] = (D)src[idx];
}

// dst[o, c] = (D) src[P[o], c]   (new order -> original order)
template <typename S, typename D>
__global__ void permute_out_kernel(int n, int R, const int32_t *__restrict__ P,
                                   const S *__restrict__ src, D *__restrict__ dst)
{
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n * R) return;
  const int o = (int)(idx / R), c = (int)(idx - (int64_t)o * R);
  dst[idx] = (D)src[(size_t)P[o] * R + c];
}

template <typename S, typename D>
__global__ void convert_kernel(int64_t count, const S *__restrict__ src, D *__restrict__ dst)
{
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < count) dst[idx] = (D)src[idx];
}

// y = a - b elementwise (count entries)
template <typename T>
__global__ void sub_kernel(int64_t count, const T *__restrict__ a, const T *__restrict__ b,
                           T *__restrict__ y)
{
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < count) y[idx] = a[idx] - b[idx];
}

// x64 += (double) d for columns whose status says they took part
template <typename T>
__global__ void accumulate_kernel(int n, int R, const T *__restrict__ d, double *__restrict__ x)
{
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < (int64_t)n * R) x[idx] += (double)d[idx];
}

// dst[i, k] = src[i, idx[k]]   (n rows, R -> Rs columns)
template <typename T>
__global__ void gather_cols_kernel(int n, int R, int Rs, const int32_t *__restrict__ idx,
                                   const T *__restrict__ src, T *__restrict__ dst)
{
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)n * Rs) return;
  const int i = (int)(t / Rs), k = (int)(t - (int64_t)i * Rs);
  dst[t] = src[(size_t)i * R + idx[k]];
}

// dst[i, idx[k]] = src[i, k]
template <typename T>
__global__ void scatter_cols_kernel(int n, int R, int Rs, const int32_t *__restrict__ idx,
                                    const T *__restrict__ src, T *__restrict__ dst)
{
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)n * Rs) return;
  const int i = (int)(t / Rs), k = (int)(t - (int64_t)i * Rs);
  dst[(size_t)i * R + idx[k]] = src[t];
}

// Column compaction of a batched PCG: the per-column state of the columns
// idx[0 .. Rs) moves to columns 0 .. Rs of dst (the iteration temporaries
// alpha, beta and p.t are recomputed; the stop flags start clear)
__global__ void gather_scalars_kernel(int Rs, const int32_t *__restrict__ idx, PcgScalars src, PcgScalars dst)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k == 0) {
    *dst.done = 0;
    *dst.want = 0;
  }
  if (k >= Rs) return;
  const int c = idx[k];
  dst.rz[k] = src.rz[c];
  dst.b2[k] = src.b2[c];
  dst.thr[k] = src.thr[c];
  dst.rr[k] = src.rr[c];
  dst.rr_ref[k] = src.rr_ref[c];
  dst.stall[k] = src.stall[c];
  dst.status[k] = src.status[c];
  dst.iters[k] = src.iters[c];
}

// ... and back: the outcome of compacted column k to column idx[k] of dst
__global__ void scatter_scalars_kernel(int Rs, const int32_t *__restrict__ idx, PcgScalars src, PcgScalars dst)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= Rs) return;
  const int c = idx[k];
  dst.rz[c] = src.rz[k];
  dst.rr[c] = src.rr[k];
  dst.rr_ref[c] = src.rr_ref[k];
  dst.stall[c] = src.stall[k];
  dst.status[c] = src.status[k];
  dst.iters[c] = src.iters[k];
}

// points (n x 3 float, stride 3) -> float4, optionally gathered by `order`
__global__ void pack_points_kernel(int n, const float *__restrict__ src,
                                   const int32_t *__restrict__ order, float4 *__restrict__ dst)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int o = order ? order[i] : i;
  dst[i] = make_float4(src[3 * (size_t)o], src[3 * (size_t)o + 1], src[3 * (size_t)o + 2], 0.f);
}

}  // namespace mbc
