// warmstart.cu -- applies a predicted warm-start correction in the basis of
// the isolated-body rigid-mode solutions.
//
// For a scene of bodies, U (n x 6) holds, on the sources of each body c, that
// body's own solution for its 6 rigid modes when it is alone (base pose).
// A correction for column block b (the 6 modes of body b) on the sources of
// body c is U[c sources] * H[c][b] with H a 6 x 6 matrix, so
//   X[j, 6b + m] += sum_k U[j, k] H[src_body[j]][b][k][m].
// No counterpart in the reference (its PCG starts from zero).
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "mbc_internal.h"

namespace {

// one thread per (source j, column); columns fastest, so a warp reads one
// row of X and the same H row block
__global__ void warm_correct_kernel(int n, int R, const int32_t *__restrict__ src_body, int nb,
                                    const float *__restrict__ U, const float *__restrict__ H,
                                    float *__restrict__ X)
{
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)n * R) return;
  const int j = (int)(t / R), col = (int)(t - (int64_t)j * R);
  const int b = col / 6, m = col - 6 * b;
  const int c = src_body[j];
  if (c < 0 || c >= nb || b >= nb) return;
  const float *h = H + ((int64_t)c * nb + b) * 36;
  const float *u = U + (int64_t)j * 6;
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 6; ++k) s = fmaf(u[k], h[k * 6 + m], s);
  X[t] += s;
}

}  // namespace

extern "C" mbc_status mbc_warm_correct(int32_t n, int32_t R, const int32_t *src_body, int32_t n_bodies,
                                       const float *U, const float *H, float *X, mbc_stream stream)
{
  if (n <= 0 || R <= 0 || n_bodies <= 0 || !src_body || !U || !H || !X)
    return mbc::fail(MBC_BAD_ARG, "mbc_warm_correct: NULL pointer or non-positive size");
  if (R > 6 * n_bodies) return mbc::fail(MBC_BAD_ARG, "mbc_warm_correct: R above 6 * n_bodies");
  const int64_t cnt = (int64_t)n * R;
  warm_correct_kernel<<<(unsigned)((cnt + 255) / 256), 256, 0, (cudaStream_t)stream>>>(n, R, src_body, n_bodies, U,
                                                                                      H, X);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return mbc::fail(MBC_CUDA_ERROR, std::string("mbc_warm_correct: ") + cudaGetErrorString(e));
  return MBC_OK;
}
