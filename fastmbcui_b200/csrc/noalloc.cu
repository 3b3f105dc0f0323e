// noalloc.cu -- the matrix-free point-kernel matvec without any device
// allocation, for callers that cannot let this library call cudaMalloc.
//
// Who needs it: a host that owns the whole device through its own memory pool
// (a simulation or rendering loop with a fixed memory budget, a framework
// whose caching allocator has already reserved the memory) and so forbids
// third-party cudaMalloc/cudaFree inside its step -- those calls can block on
// the whole device and fail late when the pool holds the memory.  The solver
// entry points allocate their workspaces on first use (mbc_apply_K and
// mbc_apply_KT among them); this one does not.
//
// The kernels are the CUDA-core point kernels of the solver (pk_rows_kernel /
// pk_cols_kernel).  Their only workspace, the coordinates packed as float4,
// lives in the file-scope device array below instead of in solver buffers.
// That array is part of this library's device image: every GPU on which the
// library's kernels are loaded holds its 4 MiB until the process exits.
#include <cstdint>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "matvec.cuh"
#include "mbc_internal.h"

namespace {

using mbc::fail;

// float4 slots of packed coordinates: [x (nf) | n_x (nf) | y (n)], each part
// starting on a 256-byte boundary.  4 MiB.
constexpr int64_t kSlots = (int64_t)1 << 18;
constexpr int kMaxDevices = 64;

__device__ __align__(256) static float4 g_noalloc_scratch[kSlots];

// Device address of g_noalloc_scratch per device.  In host code the symbol is
// only a handle for the runtime, so the address is looked up, once per device,
// with that device current.  The addresses stay cached for the process:
// cudaDeviceReset unloads the module, after which this entry point must not
// be called again in the same process.
std::mutex g_mu;
float4 *g_addr[kMaxDevices] = {};

int64_t round16(int64_t v) { return (v + 15) / 16 * 16; }

mbc_status scratch_for_current_device(float4 **out)
{
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(MBC_CUDA_ERROR, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(MBC_UNSUPPORTED, "device ordinal above 63");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(MBC_CUDA_ERROR, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    g_addr[dev] = (float4 *)p;
  }
  *out = g_addr[dev];
  return MBC_OK;
}

// rows of an n x 3 float array -> float4 (w = 0)
__global__ void pack3_kernel(int n, const float *__restrict__ src, float4 *__restrict__ dst)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = make_float4(src[3 * (size_t)i], src[3 * (size_t)i + 1], src[3 * (size_t)i + 2], 0.f);
}

constexpr int kTjRows = 128;
constexpr int kTjCols = 64;

template <int RC, int TI>
void rows(const float4 *x4, const float4 *n4, int nf, const float4 *y4, int n, float coef, int R,
          const float *v, float *w, cudaStream_t st)
{
  dim3 grid((unsigned)((nf + TI - 1) / TI), (unsigned)(((int64_t)R + RC - 1) / RC));
  mbc::pk_rows_kernel<float, RC, TI, kTjRows><<<grid, TI, 0, st>>>(x4, n4, nf, y4, n, v, R, coef, w, R, R,
                                                                  nullptr);
}

template <int RC, int TI>
void cols(const float4 *x4, const float4 *n4, int nf, const float4 *y4, int n, float coef, int R,
          const float *w, float *t, cudaStream_t st)
{
  dim3 grid((unsigned)((n + TI - 1) / TI), (unsigned)(((int64_t)R + RC - 1) / RC));
  mbc::pk_cols_kernel<float, RC, TI, kTjCols><<<grid, TI, 0, st>>>(x4, n4, nf, y4, n, w, R, coef, t, R, R,
                                                                  nullptr, nullptr, nullptr);
}

template <int RC, int TI>
void apply(int transpose, const float4 *x4, const float4 *n4, int nf, const float4 *y4, int n, float coef,
           int R, const float *in, float *out, cudaStream_t st)
{
  if (transpose) cols<RC, TI>(x4, n4, nf, y4, n, coef, R, in, out, st);
  else rows<RC, TI>(x4, n4, nf, y4, n, coef, R, in, out, st);
}

}  // namespace

extern "C" mbc_status mbc_point_apply_noalloc(int32_t transpose, int32_t nf, int32_t n, const float *x,
                                              const float *nx, const float *y, double coef, int32_t R,
                                              const float *in, float *out, mbc_stream stream)
{
  if (nf <= 0 || n <= 0 || R <= 0 || !x || !nx || !y || !in || !out)
    return fail(MBC_BAD_ARG, "mbc_point_apply_noalloc: NULL pointer or non-positive size");
  if (transpose != 0 && transpose != 1) return fail(MBC_BAD_ARG, "mbc_point_apply_noalloc: transpose must be 0 or 1");
  const int64_t need = 2 * round16(nf) + round16(n);
  if (need > kSlots)
    return fail(MBC_BAD_ARG, "mbc_point_apply_noalloc: 2*nf + n = " + std::to_string(2 * (int64_t)nf + n) +
                                 " points exceed the static scratch (2*ceil16(nf) + ceil16(n) <= " +
                                 std::to_string(kSlots) + " float4 slots, 4 MiB)");
  if (((int64_t)R + 31) / 32 > 65535) return fail(MBC_BAD_ARG, "mbc_point_apply_noalloc: R above 2,097,120");
  // the kernels read `in` while other blocks write `out` (both __restrict__):
  // an in-place or overlapping call would silently return wrong values
  const int64_t in_bytes = (int64_t)(transpose ? nf : n) * R * (int64_t)sizeof(float);
  const int64_t out_bytes = (int64_t)(transpose ? n : nf) * R * (int64_t)sizeof(float);
  const uintptr_t i0 = (uintptr_t)in, o0 = (uintptr_t)out;
  if (i0 < o0 + (uintptr_t)out_bytes && o0 < i0 + (uintptr_t)in_bytes)
    return fail(MBC_BAD_ARG, "mbc_point_apply_noalloc: in and out overlap (they must be distinct buffers)");
  // an error left pending by earlier, unrelated work is reported as such and
  // left in place, so that the launch check below sees only this call's own
  const cudaError_t prior = cudaPeekAtLastError();
  if (prior != cudaSuccess)
    return fail(MBC_CUDA_ERROR, std::string("mbc_point_apply_noalloc: an earlier CUDA error is pending (not "
                                            "cleared, nothing launched): ") + cudaGetErrorString(prior));
  float4 *base = nullptr;
  if (mbc_status s = scratch_for_current_device(&base)) return s;
  float4 *x4 = base, *n4 = base + round16(nf), *y4 = base + 2 * round16(nf);
  cudaStream_t st = (cudaStream_t)stream;
  // Every slot the matvec reads is rewritten here first: nothing depends on
  // what an earlier call left in the array.
  pack3_kernel<<<(nf + 255) / 256, 256, 0, st>>>(nf, x, x4);
  pack3_kernel<<<(nf + 255) / 256, 256, 0, st>>>(nf, nx, n4);
  pack3_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, y, y4);
  const float c = (float)coef;
  if (R == 1) apply<1, 128>(transpose, x4, n4, nf, y4, n, c, R, in, out, st);
  else if (R <= 4) apply<4, 64>(transpose, x4, n4, nf, y4, n, c, R, in, out, st);
  else if (R <= 8) apply<8, 64>(transpose, x4, n4, nf, y4, n, c, R, in, out, st);
  else if (R <= 16) apply<16, 64>(transpose, x4, n4, nf, y4, n, c, R, in, out, st);
  else apply<32, 64>(transpose, x4, n4, nf, y4, n, c, R, in, out, st);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(MBC_CUDA_ERROR, std::string("mbc_point_apply_noalloc launch: ") + cudaGetErrorString(e));
  return MBC_OK;
}
