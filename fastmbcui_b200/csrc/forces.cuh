// Added-mass reduction of a solved scene (the consumer of the strengths):
// core/KTAB_Mfs_spclf1d.py:123-128 (Ks = Q @ phi * rho) with the quadrature
// of utils/torch_utils.py:336-347 (Q rows = (s, r x s), s = area-weighted
// normal).  Per body a and generalized normal m = (n, r x n):
//   Mf[6a + m, c] = -rho_f sum_{k in body a} w_k N_m(k) phi(k, c)
// in FP64, deterministic (fixed row groups, fixed reduction order).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mbc {

// grid (n_bodies, cdiv(R, 32)); block 256 = 8 row groups x 32 columns
__global__ void __launch_bounds__(256) added_mass_kernel(const float4 *__restrict__ x4,
                                                         const float4 *__restrict__ n4,
                                                         const float *__restrict__ w,
                                                         const int32_t *__restrict__ body_ptr,
                                                         const double *__restrict__ centers,
                                                         const double *__restrict__ phi, int R,
                                                         double rho_f, double *__restrict__ Mf)
{
  __shared__ double red[8][6][32];
  const int a = blockIdx.x, lane = threadIdx.x & 31, g = threadIdx.x >> 5;
  const int c = blockIdx.y * 32 + lane;
  const double c0 = centers[3 * a], c1 = centers[3 * a + 1], c2 = centers[3 * a + 2];
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  const int k1 = body_ptr[a + 1];
  for (int k = body_ptr[a] + g; k < k1; k += 8) {
    const float4 p = x4[k], q = n4[k];
    const double r0 = (double)p.x - c0, r1 = (double)p.y - c1, r2 = (double)p.z - c2;
    const double nx = q.x, ny = q.y, nz = q.z;
    const double N[6] = {nx, ny, nz, r1 * nz - r2 * ny, r2 * nx - r0 * nz, r0 * ny - r1 * nx};
    const double ph = c < R ? phi[(size_t)k * R + c] : 0.0;
    const double wk = (double)w[k];
#pragma unroll
    for (int m = 0; m < 6; ++m) acc[m] += wk * N[m] * ph;
  }
#pragma unroll
  for (int m = 0; m < 6; ++m) red[g][m][lane] = acc[m];
  __syncthreads();
  if (threadIdx.x < 6 * 32) {
    const int m = threadIdx.x >> 5;
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) s += red[q][m][lane];
    if (c < R) Mf[(size_t)(6 * a + m) * R + c] = -rho_f * s;
  }
}

}  // namespace mbc
