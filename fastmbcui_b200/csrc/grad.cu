// Gradients of the mfs_torch operator MinvF_float_fastGrad with respect to M
// and F, in low-rank form.
//
// The reference's backward (core/mfs_torch_py/ops.py:42-58) forms
//   W = A LV (N x N, LV = VpL^T),  grad_M = -M (W + W^T) + F LV,  grad_F = M VpL
// with dense products, O(Nf N^2).  W has rank R, so the same values are
//   grad_M = (F - M A) VpL^T - (M VpL) A^T,   grad_F = M VpL:
// two skinny products G = M [A | VpL] (Nf x 2R, one pass over M) and one
// rank-2R pass that writes grad_M, O(Nf N R) in all.
//
// FP32 operands as the reference's; the skinny products accumulate each
// 32-term slice of a dot product separately and add the slices (partial
// sums of 32 terms keep the FP32 error near sqrt(N / 32) ulps).
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "mbc_internal.h"

namespace {

using mbc::fail;

constexpr int kT = 64;    // output tile 64 x 64
constexpr int kK = 32;    // inner indices staged per pass
constexpr int kThr = 256; // 16 x 16 threads, 4 x 4 outputs each

// G (nf x 2R) = M (nf x n, ldm) [A | B]   (A, B: n x R row-major)
__global__ void __launch_bounds__(kThr) grad_products_kernel(int nf, int n, int R, const float *__restrict__ M,
                                                              int64_t ldm, const float *__restrict__ A,
                                                              const float *__restrict__ B, float *__restrict__ G)
{
  __shared__ float sM[kT][kK + 1];
  __shared__ float sB[kK][kT];
  const int r0 = blockIdx.x * kT, c0 = blockIdx.y * kT, R2 = 2 * R;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  float acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.f;
  for (int k0 = 0; k0 < n; k0 += kK) {
    for (int e = threadIdx.x; e < kT * kK; e += kThr) {
      const int rr = e / kK, kk = e - rr * kK, i = r0 + rr, k = k0 + kk;
      sM[rr][kk] = (i < nf && k < n) ? M[(size_t)i * ldm + k] : 0.f;
    }
    for (int e = threadIdx.x; e < kK * kT; e += kThr) {
      const int kk = e / kT, cc = e - kk * kT, k = k0 + kk, c = c0 + cc;
      float v = 0.f;
      if (k < n && c < R2) v = c < R ? A[(size_t)k * R + c] : B[(size_t)k * R + (c - R)];
      sB[kk][cc] = v;
    }
    __syncthreads();
    float part[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) part[a][b] = 0.f;
#pragma unroll 8
    for (int kk = 0; kk < kK; ++kk) {
      float mv[4], bv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) mv[a] = sM[ty * 4 + a][kk];
#pragma unroll
      for (int b = 0; b < 4; ++b) bv[b] = sB[kk][tx * 4 + b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) part[a][b] = fmaf(mv[a], bv[b], part[a][b]);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] += part[a][b];
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int i = r0 + ty * 4 + a;
    if (i >= nf) continue;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int c = c0 + tx * 4 + b;
      if (c < R2) G[(size_t)i * R2 + c] = acc[a][b];
    }
  }
}

// out (nf x n, ldo) = [F - G1 | G2] [B | -A]^T, G = [G1 | G2] (nf x 2R)
__global__ void __launch_bounds__(kThr) grad_lowrank_kernel(int nf, int n, int R, const float *__restrict__ F,
                                                             const float *__restrict__ G, const float *__restrict__ A,
                                                             const float *__restrict__ B, float *__restrict__ out,
                                                             int64_t ldo)
{
  __shared__ float sL[kT][kK + 1];
  __shared__ float sR[kK][kT];
  const int r0 = blockIdx.x * kT, c0 = blockIdx.y * kT, R2 = 2 * R;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  float acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.f;
  for (int k0 = 0; k0 < R2; k0 += kK) {
    for (int e = threadIdx.x; e < kT * kK; e += kThr) {
      const int rr = e / kK, kk = e - rr * kK, i = r0 + rr, k = k0 + kk;
      float v = 0.f;
      if (i < nf && k < R2) v = k < R ? F[(size_t)i * R + k] - G[(size_t)i * R2 + k] : G[(size_t)i * R2 + k];
      sL[rr][kk] = v;
    }
    for (int e = threadIdx.x; e < kK * kT; e += kThr) {
      const int cc = e / kK, kk = e - cc * kK, j = c0 + cc, k = k0 + kk;
      float v = 0.f;
      if (j < n && k < R2) v = k < R ? B[(size_t)j * R + k] : -A[(size_t)j * R + (k - R)];
      sR[kk][cc] = v;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < kK; ++kk) {
      float lv[4], rv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) lv[a] = sL[ty * 4 + a][kk];
#pragma unroll
      for (int b = 0; b < 4; ++b) rv[b] = sR[kk][tx * 4 + b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = fmaf(lv[a], rv[b], acc[a][b]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int i = r0 + ty * 4 + a;
    if (i >= nf) continue;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int j = c0 + tx * 4 + b;
      if (j < n) out[(size_t)i * ldo + j] = acc[a][b];
    }
  }
}

// grad_F (nf x R) = G2
__global__ void grad_f_kernel(int nf, int R, const float *__restrict__ G, float *__restrict__ gF)
{
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)nf * R) return;
  const int i = (int)(t / R), r = (int)(t - (int64_t)i * R);
  gF[t] = G[(size_t)i * 2 * R + R + r];
}

}  // namespace

extern "C" mbc_status mbc_minvf_grad(int32_t nf, int32_t n, int32_t R, const float *M, int64_t ldm,
                                     const float *F, const float *A, const float *VpL, float *work,
                                     float *grad_M, int64_t ldg, float *grad_F, mbc_stream stream)
{
  if (nf <= 0 || n <= 0 || R <= 0 || !M || !F || !A || !VpL || !work || ldm < n)
    return fail(MBC_BAD_ARG, "mbc_minvf_grad: bad sizes or NULL input");
  if (grad_M && ldg < n) return fail(MBC_BAD_ARG, "mbc_minvf_grad: grad_M row stride below n");
  if ((nf + kT - 1) / kT > 2147483647 || (2 * (int64_t)R + kT - 1) / kT > 65535 || ((int64_t)n + kT - 1) / kT > 65535)
    return fail(MBC_BAD_ARG, "mbc_minvf_grad: sizes beyond the launch grid");
  cudaStream_t st = (cudaStream_t)stream;
  const cudaError_t prior = cudaPeekAtLastError();
  if (prior != cudaSuccess)
    return fail(MBC_CUDA_ERROR, std::string("mbc_minvf_grad: an earlier CUDA error is pending: ") +
                                    cudaGetErrorString(prior));
  grad_products_kernel<<<dim3((nf + kT - 1) / kT, (2 * R + kT - 1) / kT), kThr, 0, st>>>(nf, n, R, M, ldm, A, VpL,
                                                                                          work);
  if (grad_F) {
    const int64_t cnt = (int64_t)nf * R;
    grad_f_kernel<<<(unsigned)((cnt + 255) / 256), 256, 0, st>>>(nf, R, work, grad_F);
  }
  if (grad_M)
    grad_lowrank_kernel<<<dim3((nf + kT - 1) / kT, (n + kT - 1) / kT), kThr, 0, st>>>(nf, n, R, F, work, A, VpL,
                                                                                     grad_M, ldg);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(MBC_CUDA_ERROR, std::string("mbc_minvf_grad launch: ") + cudaGetErrorString(e));
  return MBC_OK;
}
