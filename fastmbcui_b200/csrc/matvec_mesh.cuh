// Matrix-free mesh collocation operator: K(f, j) = the solid angle of
// triangle f seen from source j (utils/torch_utils.py:306-334,
// compute_solid_angle, the matrix the reference assembles densely in torch
// every step, core/KTAB_Mfs_spclf1d.py:114):
//   K(f, j) = 2 atan2(R1 . (R2 x R3), l1 l2 l3 + (R1.R2) l3 + (R1.R3) l2 + (R2.R3) l1),
//   Rk = v_k(f) - y_j, lk = |Rk|  (van Oosterom and Strackee).
// The entries are evaluated in registers inside the matvec (and the factor's
// panels), so the Nf x N matrix is never stored.  A face's three vertices are
// three float4 row arrays (v1, v2, v3); the kernels follow the point-kernel
// ones (matvec.cuh): rows stage sources through shared memory, columns stage
// faces.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mbc {

template <typename T>
struct SolidAngle;

template <>
struct SolidAngle<double> {
  __device__ __forceinline__ static double eval(const float4 &a, const float4 &b, const float4 &c,
                                                const float4 &s)
  {
    const double ax = (double)a.x - s.x, ay = (double)a.y - s.y, az = (double)a.z - s.z;
    const double bx = (double)b.x - s.x, by = (double)b.y - s.y, bz = (double)b.z - s.z;
    const double cx = (double)c.x - s.x, cy = (double)c.y - s.y, cz = (double)c.z - s.z;
    const double num = ax * (by * cz - bz * cy) + ay * (bz * cx - bx * cz) + az * (bx * cy - by * cx);
    const double la = sqrt(ax * ax + ay * ay + az * az);
    const double lb = sqrt(bx * bx + by * by + bz * bz);
    const double lc = sqrt(cx * cx + cy * cy + cz * cz);
    const double ab = ax * bx + ay * by + az * bz;
    const double ac = ax * cx + ay * cy + az * cz;
    const double bc = bx * cx + by * cy + bz * cz;
    return 2.0 * atan2(num, la * lb * lc + ab * lc + ac * lb + bc * la);
  }
};

template <>
struct SolidAngle<float> {
  __device__ __forceinline__ static float eval(const float4 &a, const float4 &b, const float4 &c, const float4 &s)
  {
    const float ax = a.x - s.x, ay = a.y - s.y, az = a.z - s.z;
    const float bx = b.x - s.x, by = b.y - s.y, bz = b.z - s.z;
    const float cx = c.x - s.x, cy = c.y - s.y, cz = c.z - s.z;
    const float num = ax * (by * cz - bz * cy) + ay * (bz * cx - bx * cz) + az * (bx * cy - by * cx);
    const float la = sqrtf(ax * ax + ay * ay + az * az);
    const float lb = sqrtf(bx * bx + by * by + bz * bz);
    const float lc = sqrtf(cx * cx + cy * cy + cz * cz);
    const float ab = ax * bx + ay * by + az * bz;
    const float ac = ax * cx + ay * cy + az * cz;
    const float bc = bx * cx + by * cy + bz * cz;
    return 2.0f * atan2f(num, la * lb * lc + ab * lc + ac * lb + bc * la);
  }
};

// Rows: W[f, r] = coef sum_j K(f, j) V[j, r]; one face per thread, sources in
// shared-memory tiles of TJ, RC columns per launch chunk (grid.y).
template <typename T, int RC, int TI, int TJ>
__global__ void __launch_bounds__(TI) mesh_rows_kernel(
    const float4 *__restrict__ va, const float4 *__restrict__ vb, const float4 *__restrict__ vc, int nf,
    const float4 *__restrict__ ys, int n, const T *__restrict__ v, int ldv, T coef, T *__restrict__ w,
    int ldw, int R, const int *__restrict__ done)
{
  if (done && *done) return;
  __shared__ float4 sy[TJ];
  __shared__ T sv[TJ * RC];
  const int i = blockIdx.x * TI + threadIdx.x;
  const int r0 = blockIdx.y * RC;
  const int rc = min(RC, R - r0);
  const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
  const float4 a = i < nf ? va[i] : z, b = i < nf ? vb[i] : z, c = i < nf ? vc[i] : z;
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
    for (int jj = 0; jj < jm; ++jj) {
      const T k = SolidAngle<T>::eval(a, b, c, sy[jj]);
#pragma unroll
      for (int r = 0; r < RC; ++r) acc[r] = fma(k, sv[jj * RC + r], acc[r]);
    }
  }
  if (i < nf) {
#pragma unroll
    for (int r = 0; r < RC; ++r)
      if (r < rc) w[(size_t)i * ldw + r0 + r] = coef * acc[r];
  }
}

// Columns: T[j, r] = coef sum_f K(f, j) W[f, r], optionally with the PCG
// curvature partials part[blockIdx.x * R + r] = sum over the block's sources
// of p[j, r] T[j, r] (FP64), as pk_cols_kernel.
template <typename T, int RC, int TI, int TJ>
__global__ void __launch_bounds__(TI) mesh_cols_kernel(
    const float4 *__restrict__ va, const float4 *__restrict__ vb, const float4 *__restrict__ vc, int nf,
    const float4 *__restrict__ ys, int n, const T *__restrict__ wv, int ldw, T coef, T *__restrict__ t_out,
    int ldt, int R, const T *__restrict__ pdot, double *__restrict__ part, const int *__restrict__ done)
{
  if (done && *done) return;
  __shared__ float4 sa[TJ], sb[TJ], sc[TJ];
  __shared__ T sw[TJ * RC];
  __shared__ double sred[RC][TI / 32];
  const int j = blockIdx.x * TI + threadIdx.x;
  const int r0 = blockIdx.y * RC;
  const int rc = min(RC, R - r0);
  const float4 yj = j < n ? ys[j] : make_float4(0.f, 0.f, 0.f, 0.f);
  T acc[RC];
#pragma unroll
  for (int r = 0; r < RC; ++r) acc[r] = T(0);
  for (int i0 = 0; i0 < nf; i0 += TJ) {
    const int im = min(TJ, nf - i0);
    __syncthreads();
    for (int t = threadIdx.x; t < im; t += TI) {
      sa[t] = va[i0 + t];
      sb[t] = vb[i0 + t];
      sc[t] = vc[i0 + t];
    }
    for (int t = threadIdx.x; t < im * RC; t += TI) {
      const int ii = t / RC, rr = t - ii * RC;
      sw[t] = rr < rc ? wv[(size_t)(i0 + ii) * ldw + r0 + rr] : T(0);
    }
    __syncthreads();
    for (int ii = 0; ii < im; ++ii) {
      const T k = SolidAngle<T>::eval(sa[ii], sb[ii], sc[ii], yj);
#pragma unroll
      for (int r = 0; r < RC; ++r) acc[r] = fma(k, sw[ii * RC + r], acc[r]);
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

// faces (nf x 3 int32 vertex indices) -> three float4 vertex arrays; a face
// naming a vertex outside [0, n_vert) gets NaN coordinates (its row is NaN)
static __global__ void pack_faces_kernel(int nf, const float *__restrict__ V, int n_vert, const int32_t *__restrict__ F,
                                  float4 *__restrict__ va, float4 *__restrict__ vb, float4 *__restrict__ vc)
{
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  float4 *dst[3] = {va, vb, vc};
  for (int k = 0; k < 3; ++k) {
    const int v = F[3 * (size_t)f + k];
    dst[k][f] = (v >= 0 && v < n_vert)
                    ? make_float4(V[3 * (size_t)v], V[3 * (size_t)v + 1], V[3 * (size_t)v + 2], 0.f)
                    : make_float4(nanf(""), nanf(""), nanf(""), 0.f);
  }
}

}  // namespace mbc
