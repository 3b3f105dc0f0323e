// Tensor-core (tcgen05, 3xTF32) Gram assembly of the large supernodes of an
// FP32 factor:
//   Theta_s = K(:, I_s)^T K(:, I_s)   over all nf collocation rows
// (kl_chol.cu:166-223, the reference's per-supernode inner products), for
// supernodes whose row set has kMinNs <= n_s <= kMaxNs entries.  Below that
// size the contraction is too small for an M = 128 MMA and factor_kernel
// forms it on the CUDA cores; factor_kernel then runs the Cholesky and the
// KL columns of every supernode, from the Theta written here.
//
// One CTA per supernode.  The panel P = K(i0 .. i0 + 31, I_s) of a k-step is
// generated in FP32 by producer warps (the value factor_kernel's FP32 panel
// holds: coef * G), split into TF32 parts hi = rna(v), lo = rna(v - hi), and
// stored transposed, K-major with the 128-byte swizzle: operand row c is
// column c of the set, 32 rows i along K.  The same tile is the MMA's A and
// B operand, so one instruction gives a block of P^T P:
//   block 0: rows 0 .. 127 of Theta, columns 0 .. n_s (N = n_s padded to 16);
//   block 1 (n_s > 128): rows 128 .. of Theta, columns 128 .. (the rest of
//            the upper triangle; the lower-left block is its transpose);
// each as D += lo.hi + hi.lo + hi.hi (kind::tf32, K = 8 per instruction).
// The FP32 accumulation of the tensor core drops low bits with a bias, so the
// reduction over nf rows is accumulated in chunks of kChunk k-steps, each
// folded by the accumulator warps into a running sum in a second
// tensor-memory region with round-to-nearest FP32 adds (the scheme of the
// 3xTF32 matvec).  After the last chunk the accumulator warps write the
// upper triangle, mirrored, into the supernode's slice of the global Theta
// array in factor_kernel's layout (reversed order, column-major).
//
// Roles: 8 producer warps, 1 MMA warp, 4 accumulator warps.  Every mbarrier
// wait is bounded; on expiry the CTA records it in *err, stops, waits
// (bounded) for the MMAs it issued, frees its tensor memory and returns
// without writing Theta.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "matvec.cuh"
#include "matvec_mesh.cuh"
#include "matvec_tc.cuh"

namespace mbc {
namespace ftc {

constexpr int kK = 32;          // rows of the panel per k-step: one 128-byte swizzle row of TF32
constexpr int kStages = 2;      // ring of panel tiles (hi and lo)
constexpr int kChunk = 32;      // k-steps accumulated in tensor memory before a fold
constexpr int kMinNs = 32;      // smallest set the tensor path takes
constexpr int kMaxNs = 192;     // two accumulator regions of 2 x 256 columns at most
constexpr int kProducerWarps = 8;
constexpr int kMmaWarp = kProducerWarps;
constexpr int kAccWarp0 = kProducerWarps + 1;  // 4 accumulator warps
constexpr int kThreads = (kProducerWarps + 5) * 32;
constexpr int kBarAcc = 1;      // named barrier of the accumulator warps, once per chunk
constexpr int kTileRows = 256;  // operand rows per tile (two M blocks)
constexpr int kTile = kTileRows * kK * 4;  // 32 KB
constexpr int kStageBytes = 2 * kTile;     // hi, lo
constexpr int kTail = 256;
// [stages | barriers | set coordinates (float4) or dense columns]; the same
// size for every CTA, which also keeps one CTA per SM (tensor memory)
__host__ __device__ constexpr int smem_bytes() { return kStages * kStageBytes + kTail + kMaxNs * 16; }

__host__ __device__ constexpr int npad_of(int ns) { return (ns + 15) / 16 * 16; }
// columns of one accumulator region: block 0 (n_s padded) then block 1, to a multiple of 32
__host__ __device__ constexpr int region_of(int ns)
{
  return (npad_of(ns) + (npad_of(ns) > 128 ? npad_of(ns) - 128 : 0) + 31) / 32 * 32;
}
__host__ __device__ constexpr int tmem_cols_of(int ns)
{
  return 2 * region_of(ns) <= 32 ? 32 : 2 * region_of(ns) <= 64 ? 64 : 2 * region_of(ns) <= 128 ? 128
         : 2 * region_of(ns) <= 256 ? 256 : 512;
}
static_assert(2 * region_of(kMaxNs) <= 512, "accumulator regions exceed tensor memory");

struct GramArgs {
  const int32_t *list;  // supernodes of this launch (kMinNs <= n_s <= kMaxNs)
  int32_t count;
  const int32_t *set_ptr, *set_ind;
  const int64_t *th_ptr;
  int32_t kind;                // 0 dense, 1 point kernel, 2 mesh
  const float4 *xr, *nr, *zr;  // rows: points and normals, or face vertices 1, 2, 3
  const float4 *ys;            // sources, new order
  const float *M;              // dense operator
  int64_t ldm;
  const int32_t *Pinv;
  int32_t nf;
  float coef;
  float *theta;                // per supernode: n_s x n_s, reversed, column-major
  int32_t *err;                // 1 a bounded wait expired, 2 shared memory misaligned, 4 a set too large
  // polls after which a wait for a partner gives up (0: tc::kWaitLimit); the
  // wait that drains the CTA's own MMAs always uses tc::kWaitLimit
  uint32_t wait_limit;
};

__global__ void __launch_bounds__(kThreads, 1) gram_tc_kernel(GramArgs a)
{
  extern __shared__ __align__(1024) unsigned char smem[];
  if (tc::smem_u32(smem) & 1023u) {
    if (threadIdx.x == 0) atomicMax(a.err, 2);
    return;
  }
  const int s = a.list[blockIdx.x];
  const int sb = a.set_ptr[s];
  const int ns = a.set_ptr[s + 1] - sb;
  if (ns < 1 || ns > kMaxNs) {
    if (threadIdx.x == 0) atomicMax(a.err, 4);
    return;
  }
  const int npad = npad_of(ns);
  const int rcols = region_of(ns);
  const int tcols = tmem_cols_of(ns);
  const bool two = npad > 128;
  unsigned char *tail = smem + kStages * kStageBytes;
  uint64_t *afull = reinterpret_cast<uint64_t *>(tail);  // tile written by the producers
  uint64_t *aempty = afull + kStages;                    // tile read by its MMAs
  uint64_t *chunk_full = aempty + kStages;
  uint64_t *chunk_free = chunk_full + 1;
  uint64_t *mma_done = chunk_free + 1;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mma_done + 1);
  int *s_fail = reinterpret_cast<int *>(tmem_slot + 1);
  volatile int *s_aflag = s_fail + 1;  // [2]
  float4 *s_src = reinterpret_cast<float4 *>(tail + kTail);
  int32_t *s_col = reinterpret_cast<int32_t *>(tail + kTail);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nks = (a.nf + kK - 1) / kK;
  const int nchunks = (nks + kChunk - 1) / kChunk;
  const uint32_t WL = a.wait_limit ? a.wait_limit : tc::kWaitLimit;

  for (int p = tid; p < ns; p += kThreads) {
    const int c = a.set_ind[sb + p];
    if (a.kind != 0) s_src[p] = a.ys[c];
    else s_col[p] = a.Pinv[c];
  }
  if (tid == 0) {
    for (int k = 0; k < kStages; ++k) {
      tc::mbar_init(&afull[k], kProducerWarps);
      tc::mbar_init(&aempty[k], 1);
    }
    tc::mbar_init(chunk_full, 1);
    tc::mbar_init(chunk_free, 4);
    tc::mbar_init(mma_done, 1);
    *s_fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     tc::smem_u32(tmem_slot)),
                 "r"(tcols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem_acc = *tmem_slot;
  const uint32_t tmem_sum = tmem_acc + (uint32_t)rcols;
  volatile int *vfail = s_fail;

  if (warp < kProducerWarps) {
    // ---------------- producers: the transposed panel, hi and lo ----------------
    // units (operand row c, group of 4 rows i): c = unit % rows_used runs over
    // lanes; rows_used = the operand rows the MMAs read (n_s padded)
    const int rows_used = two ? kTileRows : 128;
    const int units = rows_used * (kK / 4);
    for (int ks = 0; ks < nks; ++ks) {
      const int st = ks % kStages;
      // warp-uniform decision: lane 0's view of the failure flag
      const bool got = tc::mbar_wait_warp(&aempty[st], ((ks / kStages) & 1) ^ 1, 0, WL);
      if (__shfl_sync(0xffffffffu, (!got || *vfail) ? 1 : 0, 0)) {
        if (lane == 0) *s_fail = 1;
        break;
      }
      unsigned char *Thi = smem + st * kStageBytes, *Tlo = Thi + kTile;
      const int i0 = ks * kK;
      for (int u = tid; u < units; u += kProducerWarps * 32) {
        const int c = u % rows_used, kq = u / rows_used;
        uint32_t h[4], l[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int i = i0 + kq * 4 + e;
          float v = 0.f;
          if (c < ns && i < a.nf) {
            if (a.kind == 1) v = a.coef * PointKernel<float>::eval(__ldg(a.xr + i), __ldg(a.nr + i), s_src[c]);
            else if (a.kind == 2)
              v = a.coef * SolidAngle<float>::eval(__ldg(a.xr + i), __ldg(a.nr + i), __ldg(a.zr + i), s_src[c]);
            else v = __ldg(a.M + (size_t)i * a.ldm + s_col[c]);
          }
          tc::split_tf32(v, h[e], l[e]);
        }
        const uint32_t off = tc::sw128(c, kq * 4);
        *reinterpret_cast<uint4 *>(Thi + off) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4 *>(Tlo + off) = make_uint4(l[0], l[1], l[2], l[3]);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&afull[st]);
    }
  } else if (warp == kMmaWarp) {
    // ---------------- MMA issue ----------------
    if (lane == 0) {
      const uint32_t id0 = tc::idesc_tf32(npad);
      const uint32_t id1 = two ? tc::idesc_tf32(npad - 128) : 0u;
      const uint32_t boff = 128 * 128;  // operand row 128: block 1's A and B
      for (int ks = 0; ks < nks; ++ks) {
        const int st = ks % kStages, kc = ks % kChunk;
        if (*vfail || !tc::mbar_wait_one(&afull[st], (ks / kStages) & 1, 0, WL) ||
            (kc == 0 && ks > 0 && !tc::mbar_wait_one(chunk_free, ((ks / kChunk) - 1) & 1, 0, WL))) {
          *s_fail = 1;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t Thi = tc::smem_u32(smem + st * kStageBytes), Tlo = Thi + kTile;
#pragma unroll
        for (int kk = 0; kk < kK / 8; ++kk) {
          const uint32_t ko = kk * 32;  // 8 TF32 = 32 bytes along the swizzled row
          const uint32_t acc0 = (kc > 0 || kk > 0) ? 1u : 0u;
          tc::mma_tf32(tmem_acc, tc::desc_sw128(Tlo + ko), tc::desc_sw128(Thi + ko), id0, acc0);
          tc::mma_tf32(tmem_acc, tc::desc_sw128(Thi + ko), tc::desc_sw128(Tlo + ko), id0, 1u);
          tc::mma_tf32(tmem_acc, tc::desc_sw128(Thi + ko), tc::desc_sw128(Thi + ko), id0, 1u);
          if (two) {
            const uint32_t d1 = tmem_acc + (uint32_t)npad;
            tc::mma_tf32(d1, tc::desc_sw128(Tlo + boff + ko), tc::desc_sw128(Thi + boff + ko), id1, acc0);
            tc::mma_tf32(d1, tc::desc_sw128(Thi + boff + ko), tc::desc_sw128(Tlo + boff + ko), id1, 1u);
            tc::mma_tf32(d1, tc::desc_sw128(Thi + boff + ko), tc::desc_sw128(Thi + boff + ko), id1, 1u);
          }
        }
        tc::mma_commit(&aempty[st]);
        if (kc == kChunk - 1 || ks == nks - 1) tc::mma_commit(chunk_full);
      }
      // after a failure, release the accumulator warps once every MMA issued
      // so far has finished; tensor memory is freed only after that point
      if (*vfail) tc::mma_commit(chunk_full);
      tc::mma_commit(mma_done);
      if (!tc::mbar_wait_one(mma_done, 0)) *s_fail = 1;
    }
  } else {
    // ---------------- accumulator warps: fold chunks, then Theta ----------------
    const int q = warp & 3;  // tensor-memory lane quarter of this warp
    const uint32_t lane_off = (uint32_t)(q * 32) << 16;
    float *A = a.theta + a.th_ptr[s];
    bool ok = true;
    for (int c = 0; c < nchunks; ++c) {
      if (warp == kAccWarp0 && lane == 0) s_aflag[c & 1] = tc::mbar_wait_one(chunk_full, c & 1, 64, WL) ? 1 : 0;
      asm volatile("bar.sync %0, 128;" ::"n"(kBarAcc) : "memory");
      // only the flag the polling lane set before the barrier decides here,
      // so that all four warps take the same branch (a warp that left alone
      // would strand the others at the named barrier)
      if (!s_aflag[c & 1]) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const bool last = c == nchunks - 1;
      // no barrier follows the last chunk; the tensor-memory loads below are
      // warp-collective, so lane 0's view decides for its warp
      if (last && __shfl_sync(0xffffffffu, *vfail, 0)) {
        ok = false;
        break;
      }
      for (int c0 = 0; c0 < rcols; c0 += 32) {
        float v[32];
        tc::tmem_ld32(tmem_acc + lane_off + (uint32_t)c0, v);
        if (c > 0) {
          float u[32];
          tc::tmem_ld32(tmem_sum + lane_off + (uint32_t)c0, u);
#pragma unroll
          for (int k = 0; k < 32; ++k) v[k] += u[k];
        }
        if (!last) {
          tc::tmem_st32(tmem_sum + lane_off + (uint32_t)c0, v);
          continue;
        }
        // Theta(m, n), m <= n, and its mirror; column col of the region is
        // block 0's column col, or block 1's column 128 + col - npad
#pragma unroll
        for (int k = 0; k < 32; ++k) {
          const int col = c0 + k;
          int m, n;
          if (col < npad) {
            m = q * 32 + lane;
            n = col;
          } else {
            m = 128 + q * 32 + lane;
            n = 128 + col - npad;
          }
          if (m < ns && n < ns && m <= n) {
            const int rm = ns - 1 - m, rn = ns - 1 - n;
            A[rm + (size_t)rn * ns] = v[k];
            A[rn + (size_t)rm * ns] = v[k];
          }
        }
      }
      if (!last) {
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(chunk_free);
      }
    }
    if (!ok) *s_fail = 1;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (tid == 0 && *s_fail && a.err) atomicMax(a.err, 1);
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_acc), "r"(tcols) : "memory");
  }
}

}  // namespace ftc
}  // namespace mbc
