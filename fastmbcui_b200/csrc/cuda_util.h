// Error-checking macros and launch helpers shared by the solver's CUDA
// translation units (each returns an mbc_status from the enclosing function).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "mbc_internal.h"

namespace mbc {

#define MBC_CK(call)                                                                      \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return fail(MBC_CUDA_ERROR, std::string(#call) + ": " + cudaGetErrorString(e_));     \
  } while (0)

#define MBC_CKL()                                                                         \
  do {                                                                                     \
    cudaError_t e_ = cudaGetLastError();                                                   \
    if (e_ != cudaSuccess)                                                                 \
      return fail(MBC_CUDA_ERROR, std::string("kernel launch: ") + cudaGetErrorString(e_)); \
  } while (0)

#define MBC_TRY(expr)              \
  do {                             \
    mbc_status s_ = (expr);        \
    if (s_ != MBC_OK) return s_;   \
  } while (0)

inline unsigned cdiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

// Opt a kernel in to the device's largest dynamic shared memory.  The limit
// is per-kernel state shared by every host thread; setting it to one fixed
// value (rather than to each launch's own size) keeps concurrent solvers
// from lowering it under one another's launches.
template <typename K>
mbc_status allow_max_smem(K kern, size_t need)
{
  int dev = 0, cap = 0;
  MBC_CK(cudaGetDevice(&dev));
  MBC_CK(cudaDeviceGetAttribute(&cap, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa;
  MBC_CK(cudaFuncGetAttributes(&fa, kern));
  const int dyn_cap = cap - (int)fa.sharedSizeBytes;  // static + dynamic <= the opt-in cap
  if (need > (size_t)std::max(dyn_cap, 0))
    return fail(MBC_UNSUPPORTED, "kernel needs " + std::to_string(need) + " B of dynamic shared memory, device allows " +
                                     std::to_string(dyn_cap));
  MBC_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_cap));
  return MBC_OK;
}

}  // namespace mbc
