// Matvec kernels for the MFS operator K (nf collocation rows x n sources).
//
//  * point kernel, evaluated in registers:
//      K(i,j) = coef ((x_i - y_j).n_i) / |x_i - y_j|^3   (src/kernels.h:24-40)
//    rows   : W[i, r] = sum_j K(i,j) V[j, r]   (one row per thread, sources
//             staged through shared memory in tiles, R columns per chunk)
//    columns: T[j, r] = sum_i K(i,j) W[i, r]   (one source per thread, rows
//             staged through shared memory)
//  * dense caller matrix M (row-major float32), the mfs_torch operator input:
//    rows   : warp per row, float4 loads of M, warp-shuffle reduction;
//    columns: thread per column, coalesced over consecutive columns.
//
// Coordinates are float4 (x, y, z, 0) so every point is one 16-byte load.
// Vectors are row-major with leading dimension `ld` (the RHS count R); a
// launch handles columns [r0, r0 + RC).  T is the arithmetic type.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mbc {

// Reciprocal square root to FP64 accuracy: FP32 hardware estimate refined by
// two Newton-Raphson steps y <- y (3 - a y^2) / 2, written as
// e = 1 - a y^2 (one FMA), y <- y + (y/2) e.  Valid for a in FP32 range.
__device__ __forceinline__ double rsqrt_nr(double a)
{
  double y = (double)rsqrtf((float)a);
  double e = fma(-a * y, y, 1.0);
  y = fma(0.5 * y, e, y);
  e = fma(-a * y, y, 1.0);
  return fma(0.5 * y, e, y);
}

template <typename T>
struct PointKernel;

template <>
struct PointKernel<float> {
  __device__ __forceinline__ static float eval(const float4 &x, const float4 &nx, const float4 &y)
  {
    const float dx = x.x - y.x, dy = x.y - y.y, dz = x.z - y.z;
    const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    const float ir = rsqrtf(r2);
    const float rn = fmaf(dz, nx.z, fmaf(dy, nx.y, dx * nx.x));
    return rn * (ir * ir * ir);
  }
};

template <>
struct PointKernel<double> {
  __device__ __forceinline__ static double eval(const float4 &x, const float4 &nx, const float4 &y)
  {
    const double dx = (double)x.x - (double)y.x, dy = (double)x.y - (double)y.y,
                 dz = (double)x.z - (double)y.z;
    const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
    const double ir = rsqrt_nr(r2);
    const double rn = fma(dz, (double)nx.z, fma(dy, (double)nx.y, dx * (double)nx.x));
    return rn * (ir * ir * ir);
  }
};

// Single-layer potential kernel 1/|x - y| in FP64 (the normal is unused):
// the potential of the solved strengths, utils/torch_utils.py:254-276.
struct SingleLayer64 {
  __device__ __forceinline__ static double eval(const float4 &x, const float4 &, const float4 &y)
  {
    const double dx = (double)x.x - (double)y.x, dy = (double)x.y - (double)y.y,
                 dz = (double)x.z - (double)y.z;
    return rsqrt_nr(fma(dz, dz, fma(dy, dy, dx * dx)));
  }
};

// Rows direction.  Block = TI threads, one row each; grid.x over rows,
// grid.y over RC-column chunks.  `done` (may be NULL) lets an iteration that
// has nothing left to do exit at once.
template <typename T, int RC, int TI, int TJ, class Ker = PointKernel<T>>
__global__ void __launch_bounds__(TI) pk_rows_kernel(
    const float4 *__restrict__ xr, const float4 *__restrict__ nr, int nf,
    const float4 *__restrict__ ys, int n, const T *__restrict__ v, int ldv,
    T coef, T *__restrict__ w, int ldw, int R, const int *__restrict__ done)
{
  if (done && *done) return;
  __shared__ float4 sy[TJ];
  __shared__ T sv[TJ * RC];
  const int i = blockIdx.x * TI + threadIdx.x;
  const int r0 = blockIdx.y * RC;
  const int rc = min(RC, R - r0);
  float4 xi = make_float4(0.f, 0.f, 0.f, 0.f), ni = xi;
  if (i < nf) {
    xi = xr[i];
    ni = nr[i];
  }
  T acc[RC];
#pragma unroll
  for (int r = 0; r < RC; ++r) acc[r] = T(0);
  for (int j0 = 0; j0 < n; j0 += TJ) {
    const int jm = min(TJ, n - j0);
    __syncthreads();
    for (int t = threadIdx.x; t < jm; t += TI) sy[t] = ys[j0 + t];
    for (int t = threadIdx.x; t < jm * RC; t += TI) {
      const int jj = t / RC, rr = t - jj * RC;
      sv[t] = rr < rc ? v[(size_t)(j0 + jj) * ldv + r0 + rr] : T(0);
    }
    __syncthreads();
    if (jm == TJ) {
#pragma unroll 2
      for (int jj = 0; jj < TJ; ++jj) {
        const T k = Ker::eval(xi, ni, sy[jj]);
#pragma unroll
        for (int r = 0; r < RC; ++r) acc[r] = fma(k, sv[jj * RC + r], acc[r]);
      }
    } else {
      for (int jj = 0; jj < jm; ++jj) {
        const T k = Ker::eval(xi, ni, sy[jj]);
#pragma unroll
        for (int r = 0; r < RC; ++r) acc[r] = fma(k, sv[jj * RC + r], acc[r]);
      }
    }
  }
  if (i < nf) {
#pragma unroll
    for (int r = 0; r < RC; ++r)
      if (r < rc) w[(size_t)i * ldw + r0 + r] = coef * acc[r];
  }
}

// Columns direction: T[j, r] = coef * sum_i K(i,j) W[i, r].  Optionally fused
// with the PCG curvature partial sums: part[blockIdx.x * R + r] =
// sum over this block's sources of p[j, r] * T[j, r] (FP64).
template <typename T, int RC, int TI, int TJ>
__global__ void __launch_bounds__(TI) pk_cols_kernel(
    const float4 *__restrict__ xr, const float4 *__restrict__ nr, int nf,
    const float4 *__restrict__ ys, int n, const T *__restrict__ wv, int ldw,
    T coef, T *__restrict__ t_out, int ldt, int R, const T *__restrict__ pdot,
    double *__restrict__ part, const int *__restrict__ done)
{
  if (done && *done) return;
  __shared__ float4 sx[TJ], sn[TJ];
  __shared__ T sw[TJ * RC];
  __shared__ double sred[RC][TI / 32];
  const int j = blockIdx.x * TI + threadIdx.x;
  const int r0 = blockIdx.y * RC;
  const int rc = min(RC, R - r0);
  float4 yj = make_float4(0.f, 0.f, 0.f, 0.f);
  if (j < n) yj = ys[j];
  T acc[RC];
#pragma unroll
  for (int r = 0; r < RC; ++r) acc[r] = T(0);
  for (int i0 = 0; i0 < nf; i0 += TJ) {
    const int im = min(TJ, nf - i0);
    __syncthreads();
    for (int t = threadIdx.x; t < im; t += TI) {
      sx[t] = xr[i0 + t];
      sn[t] = nr[i0 + t];
    }
    for (int t = threadIdx.x; t < im * RC; t += TI) {
      const int ii = t / RC, rr = t - ii * RC;
      sw[t] = rr < rc ? wv[(size_t)(i0 + ii) * ldw + r0 + rr] : T(0);
    }
    __syncthreads();
    if (im == TJ) {
#pragma unroll 2
      for (int ii = 0; ii < TJ; ++ii) {
        const T k = PointKernel<T>::eval(sx[ii], sn[ii], yj);
#pragma unroll
        for (int r = 0; r < RC; ++r) acc[r] = fma(k, sw[ii * RC + r], acc[r]);
      }
    } else {
      for (int ii = 0; ii < im; ++ii) {
        const T k = PointKernel<T>::eval(sx[ii], sn[ii], yj);
#pragma unroll
        for (int r = 0; r < RC; ++r) acc[r] = fma(k, sw[ii * RC + r], acc[r]);
      }
    }
  }
#pragma unroll
  for (int r = 0; r < RC; ++r) acc[r] *= coef;
  if (j < n) {
#pragma unroll
    for (int r = 0; r < RC; ++r)
      if (r < rc) t_out[(size_t)j * ldt + r0 + r] = acc[r];
  }
  if (part) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int r = 0; r < RC; ++r) {
      double d = 0.0;
      if (j < n && r < rc) d = (double)pdot[(size_t)j * ldt + r0 + r] * (double)acc[r];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
      if (lane == 0) sred[r][wid] = d;
    }
    __syncthreads();
    if (threadIdx.x < RC && threadIdx.x < rc) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < TI / 32; ++k) s += sred[threadIdx.x][k];
      part[(size_t)blockIdx.x * R + r0 + threadIdx.x] = s;
    }
  }
}

// Dense rows: W[i, r] = sum_o M[i, o] Vnew[P[o], r].  One warp per row.
template <typename T, int RC>
__global__ void __launch_bounds__(256) dense_rows_kernel(
    const float *__restrict__ M, int64_t ldm, int nf, int n, const int *__restrict__ P,
    const T *__restrict__ v, int ldv, T *__restrict__ w, int ldw, int R,
    const int *__restrict__ done)
{
  if (done && *done) return;
  const int warps = blockDim.x >> 5;
  const int i = blockIdx.x * warps + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  const int r0 = blockIdx.y * RC;
  const int rc = min(RC, R - r0);
  if (i >= nf) return;
  const float *row = M + (size_t)i * ldm;
  T acc[RC];
#pragma unroll
  for (int r = 0; r < RC; ++r) acc[r] = T(0);
  for (int o = lane; o < n; o += 32) {
    const T m = (T)__ldg(row + o);
    const T *vp = v + (size_t)__ldg(P + o) * ldv + r0;
#pragma unroll
    for (int r = 0; r < RC; ++r)
      if (r < rc) acc[r] = fma(m, vp[r], acc[r]);
  }
#pragma unroll
  for (int r = 0; r < RC; ++r) {
    T s = acc[r];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    acc[r] = s;
  }
  if (lane == 0) {
#pragma unroll
    for (int r = 0; r < RC; ++r)
      if (r < rc) w[(size_t)i * ldw + r0 + r] = acc[r];
  }
}

// Dense columns: Tnew[P[o], r] = sum_i M[i, o] W[i, r]; thread per column o,
// rows of W staged in shared memory.  Fused curvature partials as above.
template <typename T, int RC, int TI, int TJ>
__global__ void __launch_bounds__(TI) dense_cols_kernel(
    const float *__restrict__ M, int64_t ldm, int nf, int n, const int *__restrict__ P,
    const T *__restrict__ wv, int ldw, T *__restrict__ t_out, int ldt, int R,
    const T *__restrict__ pdot, double *__restrict__ part, const int *__restrict__ done)
{
  if (done && *done) return;
  __shared__ T sw[TJ * RC];
  __shared__ double sred[RC][TI / 32];
  const int o = blockIdx.x * TI + threadIdx.x;
  const int r0 = blockIdx.y * RC;
  const int rc = min(RC, R - r0);
  T acc[RC];
#pragma unroll
  for (int r = 0; r < RC; ++r) acc[r] = T(0);
  for (int i0 = 0; i0 < nf; i0 += TJ) {
    const int im = min(TJ, nf - i0);
    __syncthreads();
    for (int t = threadIdx.x; t < im * RC; t += TI) {
      const int ii = t / RC, rr = t - ii * RC;
      sw[t] = rr < rc ? wv[(size_t)(i0 + ii) * ldw + r0 + rr] : T(0);
    }
    __syncthreads();
    if (o < n) {
      for (int ii = 0; ii < im; ++ii) {
        const T m = (T)__ldg(M + (size_t)(i0 + ii) * ldm + o);
#pragma unroll
        for (int r = 0; r < RC; ++r) acc[r] = fma(m, sw[ii * RC + r], acc[r]);
      }
    }
  }
  const int jn = o < n ? __ldg(P + o) : 0;
  if (o < n) {
#pragma unroll
    for (int r = 0; r < RC; ++r)
      if (r < rc) t_out[(size_t)jn * ldt + r0 + r] = acc[r];
  }
  if (part) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int r = 0; r < RC; ++r) {
      double d = 0.0;
      if (o < n && r < rc) d = (double)pdot[(size_t)jn * ldt + r0 + r] * (double)acc[r];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) d += __shfl_xor_sync(0xffffffffu, d, off);
      if (lane == 0) sred[r][wid] = d;
    }
    __syncthreads();
    if (threadIdx.x < RC && threadIdx.x < rc) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < TI / 32; ++k) s += sred[threadIdx.x][k];
      part[(size_t)blockIdx.x * R + r0 + threadIdx.x] = s;
    }
  }
}

}  // namespace mbc

