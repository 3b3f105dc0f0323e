// Tensor-core (tcgen05) form of the batched point-kernel matvec.
//
//   rows:    W[i, r] = coef sum_j G(x_i, n_i, y_j) V[j, r]   (M = rows,    K = sources)
//   columns: T[j, r] = coef sum_i G(x_i, n_i, y_j) W[i, r]   (M = sources, K = rows)
//
// G = ((x - y).n) / |x - y|^3 is generated by SIMT warps tile by tile and
// never stored; the vector block is the MMA's B operand.  Accuracy is FP32
// level through "3xTF32": every operand value v is split into TF32 parts
// hi = rna(v), lo = rna(v - hi), and D += A_lo B_hi + A_hi B_lo + A_hi B_hi
// (the products are exact).  The tensor core's FP32 accumulation drops low
// bits with a bias, so an accumulator that absorbs the whole reduction
// drifts linearly with its length (measured: 2e-4 relative after 40000
// terms, against 4e-6 for round-to-nearest FMAs).  The reduction is therefore
// accumulated in chunks of kChunk k-steps: accumulator warps fold each
// finished chunk into a second tensor-memory region with round-to-nearest
// FP32 adds, which keeps the error at the level of an FP32 FMA loop.
//
// Per launch:
//   pack_b_kernel: the vector block, split into hi / lo and laid out per
//     k-step exactly as the shared-memory image the MMA reads (K-major,
//     128-byte swizzle), so a stage is one contiguous bulk copy.
//   pk_tc_kernel: one CTA owns 128 outputs (accumulator of 128 lanes x np
//     columns in tensor memory; np = R padded to 16) and walks the k-steps of
//     32 through two shared-memory rings: 2 stages of A (the G tile, hi and
//     lo) and 3 stages (2 when np > 192) of B image + coordinates, so the bulk
//     copy of a step is issued two MMA steps before it is needed:
//       loader warp  -- waits "bempty", bulk-copies the stage's coordinates
//                       and B image (cp.async.bulk, completion on "bfull");
//       16 producer warps -- wait "bfull" and "aempty", evaluate the 128 x 32
//                       tile of G in FP32 from the staged coordinates, split,
//                       store A hi / lo swizzled, fence to the async proxy,
//                       arrive on "afull";
//       MMA warp     -- waits "afull" and "bfull" (and, at a chunk start,
//                       "chunk_free"), issues 4 x 3 tcgen05.mma (kind::tf32,
//                       K = 8), commits to "aempty" and "bempty" and, at a
//                       chunk end, "chunk_full";
//       4 accumulator warps -- wait "chunk_full" (sleeping between polls),
//                       add the chunk into the running sum (tcgen05.ld / st),
//                       arrive "chunk_free"; after the last chunk they scale
//                       by coef and store, and in the columns direction form
//                       the PCG curvature partials p.t per CTA.
// Every mbarrier wait is bounded: on expiry the kernel records the failure in
// *err, stops waiting, releases the waiters it feeds, waits (bounded) for its
// own copies, frees its tensor memory and returns.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "matvec.cuh"

namespace mbc {
namespace tc {

constexpr int kM = 128;     // MMA M (outputs per CTA)
constexpr int kK = 32;      // k-step: one 128-byte swizzle row of TF32
constexpr int kAStages = 2;     // ring of produced A (G) tiles
constexpr int kMaxBStages = 3;  // ring of bulk-copied B image + coordinates
constexpr int kChunk = 32;  // k-steps accumulated in tensor memory before a fold
constexpr int kProducerWarps = 16;
constexpr int kLoaderWarp = kProducerWarps;
constexpr int kMmaWarp = kProducerWarps + 1;
constexpr int kAccWarp0 = kProducerWarps + 2;  // 4 accumulator warps
constexpr int kSchedWarp = kProducerWarps + 6;
constexpr int kThreads = (kProducerWarps + 7) * 32;
// named barriers (0 is __syncthreads).  Every participant uses bar.sync, so
// no role can run more than one step ahead of a partner.
constexpr int kBarGo = 1;      // producers + scheduler warp, once per k-step
constexpr int kBarAReady = 2;  // producers + MMA warp, once per k-step
constexpr int kBarAcc = 3;     // the 4 accumulator warps, once per chunk
constexpr int kGoCount = (kProducerWarps + 1) * 32;
constexpr int kKPerProducer = kK / (kProducerWarps / 4);  // k values per row per k-step
constexpr uint32_t kWaitLimit = 1u << 22;  // polls of a bounded wait
constexpr int kSmemLimit = 232448;        // opt-in dynamic shared memory per CTA (227 KB)
constexpr int kTail = 256 + 8192;         // barriers, then the accumulator warps' partials

constexpr int kTileA = kM * kK * 4;  // one A operand tile: 16 KB
constexpr int kABytes = kAStages * 2 * kTileA;

__host__ __device__ constexpr int tile_b_bytes(int np) { return np * kK * 4; }
__host__ __device__ constexpr int coord_bytes(int dir) { return dir == 0 ? kK * 16 : kK * 32; }
// one B stage: [B hi | B lo | coordinates], rounded so every tile stays 1024-aligned
__host__ __device__ constexpr int bstage_bytes(int np, int dir)
{
  return (2 * tile_b_bytes(np) + coord_bytes(dir) + 1023) / 1024 * 1024;
}
__host__ __device__ constexpr int b_stages(int np, int dir)
{
  return kABytes + kMaxBStages * bstage_bytes(np, dir) + kTail <= kSmemLimit ? kMaxBStages : 2;
}
// [A ring | B ring | tail]; the dynamic shared window starts 1024-aligned
__host__ __device__ constexpr int smem_bytes(int np, int dir)
{
  return kABytes + b_stages(np, dir) * bstage_bytes(np, dir) + kTail;
}

__host__ __device__ constexpr int tmem_cols_for(int np)
{
  return np <= 32 ? 32 : np <= 64 ? 64 : np <= 128 ? 128 : 256;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
  return (uint32_t)__cvta_generic_to_shared(p);
}

// byte offset of element (row, k) in a K-major, 128B-swizzled tile whose rows
// are 32 TF32 values (128 B); tiles are 1024-byte aligned
__host__ __device__ __forceinline__ uint32_t sw128(int row, int k)
{
  return (uint32_t)((row >> 3) * 1024 + (row & 7) * 128 + ((((k >> 2) ^ (row & 7)) & 7) << 4) +
                    ((k & 3) << 2));
}

__device__ __forceinline__ uint32_t tf32_rna(float v)
{
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
  return r;
}

__device__ __forceinline__ void split_tf32(float v, uint32_t &hi, uint32_t &lo)
{
  hi = tf32_rna(v);
  lo = tf32_rna(v - __uint_as_float(hi));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(uint64_t *bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// bounded wait for the phase with the given parity; false on expiry after
// `limit` polls.  Roles that wait long (sleep_ns > 0) back off between polls
// so that their polling does not take issue slots from the producer warps.
__device__ __forceinline__ bool mbar_wait_one(uint64_t *bar, uint32_t parity, uint32_t sleep_ns = 0,
                                              uint32_t limit = kWaitLimit)
{
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < limit; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
    if (sleep_ns) __nanosleep(sleep_ns);
  }
  return false;
}

// warp-uniform bounded wait: lane 0 polls, the outcome is broadcast and
// __syncwarp orders the other lanes after lane 0's acquire
__device__ __forceinline__ bool mbar_wait_warp(uint64_t *bar, uint32_t parity, uint32_t sleep_ns = 0,
                                               uint32_t limit = kWaitLimit)
{
  int got = 0;
  if ((threadIdx.x & 31) == 0) got = mbar_wait_one(bar, parity, sleep_ns, limit) ? 1 : 0;
  got = __shfl_sync(0xffffffffu, got, 0);
  __syncwarp();
  return got != 0;
}

// global -> shared bulk copy completing on an mbarrier (16-byte aligned, size % 16 == 0)
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__host__ __device__ __forceinline__ constexpr uint64_t desc_sw128(uint32_t saddr)
{
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);  // start address
  d |= (uint64_t)1 << 16;                            // LBO (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;                  // SBO: 8 rows x 128 B
  d |= (uint64_t)1 << 46;                            // descriptor version (sm100)
  d |= (uint64_t)2 << 61;                            // SWIZZLE_128B
  return d;
}

// kind::tf32, FP32 accumulate, A and B K-major, M = 128, N = np
__host__ __device__ __forceinline__ constexpr uint32_t idesc_tf32(int np)
{
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(np >> 3) << 17) | ((uint32_t)(kM >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
        "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
        "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ void tmem_st32(uint32_t taddr, const float (&v)[32])
{
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
      "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
      "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
      "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
      "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
      "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
      "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
      "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
      "r"(__float_as_uint(v[15])), "r"(__float_as_uint(v[16])), "r"(__float_as_uint(v[17])),
      "r"(__float_as_uint(v[18])), "r"(__float_as_uint(v[19])), "r"(__float_as_uint(v[20])),
      "r"(__float_as_uint(v[21])), "r"(__float_as_uint(v[22])), "r"(__float_as_uint(v[23])),
      "r"(__float_as_uint(v[24])), "r"(__float_as_uint(v[25])), "r"(__float_as_uint(v[26])),
      "r"(__float_as_uint(v[27])), "r"(__float_as_uint(v[28])), "r"(__float_as_uint(v[29])),
      "r"(__float_as_uint(v[30])), "r"(__float_as_uint(v[31]))
      : "memory");
}

// The B image: for each k-step ks, [hi tile | lo tile], each np rows x 128 B
// laid out by sw128; element (r, k) = vin[(32 ks + k) * R + r], zero outside.
// One thread per (k-step, row r, group of 4 k).  Internal linkage: several
// translation units include this header.
static __global__ void pack_b_kernel(const float *__restrict__ vin, int K_total, int R, int np, int nks,
                              uint4 *__restrict__ img, const int32_t *__restrict__ done)
{
  if (done && *done) return;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t per_ks = (int64_t)np * (kK / 4);
  if (t >= per_ks * nks) return;
  const int ks = (int)(t / per_ks);
  const int rem = (int)(t - (int64_t)ks * per_ks);
  const int r = rem % np, kq = rem / np;
  uint32_t h[4], l[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int gk = ks * kK + kq * 4 + e;
    const float v = (r < R && gk < K_total) ? vin[(size_t)gk * R + r] : 0.f;
    split_tf32(v, h[e], l[e]);
  }
  unsigned char *base = reinterpret_cast<unsigned char *>(img) + (size_t)ks * 2 * tile_b_bytes(np);
  const uint32_t off = sw128(r, kq * 4);
  *reinterpret_cast<uint4 *>(base + off) = make_uint4(h[0], h[1], h[2], h[3]);
  *reinterpret_cast<uint4 *>(base + tile_b_bytes(np) + off) = make_uint4(l[0], l[1], l[2], l[3]);
}

struct TcArgs {
  const float4 *xr, *nr;  // collocation rows (original order), padded to 32
  const float4 *ys;       // sources (new order), padded to 32
  int nf, n;
  const uint4 *bimg;      // packed B image of the input block
  float *out;             // rows: W (nf x R); columns: T (n x R)
  int R, np;              // columns and padded MMA N (multiple of 16, <= 256)
  int tmem_cols;          // per region: power of two >= np, >= 32
  float coef;
  const float *pdot;      // columns: p (n x R) for the curvature partials, or NULL
  double *part;           // columns: per-CTA partials (gridDim.x x R)
  const int32_t *done;    // PCG all-stopped flag (may be NULL)
  int32_t *err;           // 1: a bounded wait expired; 2: shared memory misaligned
  // polls after which a wait for a partner gives up (0: kWaitLimit); the
  // waits that drain the CTA's own copies and MMAs always use kWaitLimit
  uint32_t wait_limit;
};

template <int DIR>
__global__ void __launch_bounds__(kThreads, 1) pk_tc_kernel(TcArgs a)
{
  if (a.done && *a.done) return;
  extern __shared__ __align__(1024) unsigned char smem[];
  if (smem_u32(smem) & 1023u) {
    if (threadIdx.x == 0) atomicExch(a.err, 2);
    return;
  }
  const int nbs = b_stages(a.np, DIR);
  const int bst = bstage_bytes(a.np, DIR);
  const int btile = tile_b_bytes(a.np);
  unsigned char *bring = smem + kABytes;
  unsigned char *tail = bring + nbs * bst;
  uint64_t *bfull = reinterpret_cast<uint64_t *>(tail);  // B stage landed
  uint64_t *bempty = bfull + kMaxBStages;                 // B stage read by its MMAs
  uint64_t *afull = bempty + kMaxBStages;                 // A stage written by the producers
  uint64_t *aempty = afull + kAStages;                    // A stage read by its MMAs
  uint64_t *chunk_full = aempty + kAStages;
  uint64_t *chunk_free = chunk_full + 1;
  uint64_t *mma_done = chunk_free + 1;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mma_done + 1);
  int *s_fail = reinterpret_cast<int *>(tmem_slot + 1);
  volatile int *s_aflag = s_fail + 1;  // [2]: chunk landed, as seen by the polling accumulator warp
  double *s_red = reinterpret_cast<double *>(tail + 256);  // [4][R]

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int M_total = DIR == 0 ? a.nf : a.n;
  const int K_total = DIR == 0 ? a.n : a.nf;
  const int m0 = blockIdx.x * kM;
  const int nks = (K_total + kK - 1) / kK;
  const int nchunks = (nks + kChunk - 1) / kChunk;
  const int tcols = 2 * a.tmem_cols;  // [chunk accumulator | running sum]
  const uint32_t WL = a.wait_limit ? a.wait_limit : kWaitLimit;

  if (tid == 0) {
    for (int s = 0; s < kMaxBStages; ++s) {
      mbar_init(&bfull[s], 1);
      mbar_init(&bempty[s], 1);
    }
    for (int s = 0; s < kAStages; ++s) {
      mbar_init(&afull[s], kProducerWarps);
      mbar_init(&aempty[s], 1);
    }
    mbar_init(chunk_full, 1);
    mbar_init(chunk_free, 4);
    mbar_init(mma_done, 1);
    *s_fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(tcols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem_acc = *tmem_slot;
  const uint32_t tmem_sum = tmem_acc + (uint32_t)a.tmem_cols;

  // Producers never poll an mbarrier: the scheduler warp polls "bfull" and
  // "aempty" for step ks while the producers compute step ks - 1, and meets
  // them at the "go" barrier; finished A stages reach the MMA warp through the
  // "A ready" barrier.  Named barriers cannot time out, so every role takes all
  // nks steps of its barrier sequence even after a failure (s_fail), doing no
  // work in those steps.
  volatile int *vfail = s_fail;
  if (warp < kProducerWarps) {
    // ---------------- producers: the G tile ----------------
    // row 32*(warp%4) + lane, kKPerProducer values of each k-step
    const int row = (warp & 3) * 32 + lane;
    const int kbeg = (warp >> 2) * kKPerProducer;
    const int gm = m0 + row;
    float4 own = make_float4(0.f, 0.f, 0.f, 0.f), own_n = own;
    if (gm < M_total) {
      if (DIR == 0) {
        own = a.xr[gm];
        own_n = a.nr[gm];
      } else {
        own = a.ys[gm];
      }
    }
    for (int ks = 0; ks < nks; ++ks) {
      const int sa = ks % kAStages, sb = ks % nbs;
      asm volatile("bar.sync %0, %1;" ::"n"(kBarGo), "n"(kGoCount) : "memory");
      if (!*vfail) {
        unsigned char *Ahi = smem + sa * 2 * kTileA, *Alo = Ahi + kTileA;
        const float4 *co = reinterpret_cast<const float4 *>(bring + sb * bst + 2 * btile);
        const int k0 = ks * kK;
#pragma unroll
        for (int q = 0; q < kKPerProducer / 4; ++q) {
          uint32_t h[4], l[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int k = kbeg + q * 4 + e;
            float g = 0.f;
            if (gm < M_total && k0 + k < K_total) {
              if (DIR == 0) g = PointKernel<float>::eval(own, own_n, co[k]);
              else g = PointKernel<float>::eval(co[k], co[kK + k], own);
            }
            split_tf32(g, h[e], l[e]);
          }
          const uint32_t off = sw128(row, kbeg + q * 4);
          *reinterpret_cast<uint4 *>(Ahi + off) = make_uint4(h[0], h[1], h[2], h[3]);
          *reinterpret_cast<uint4 *>(Alo + off) = make_uint4(l[0], l[1], l[2], l[3]);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      }
      asm volatile("bar.sync %0, %1;" ::"n"(kBarAReady), "n"(kGoCount) : "memory");
    }
  } else if (warp == kSchedWarp) {
    // ---------------- scheduler: releases the producers step by step ----------------
    for (int ks = 0; ks < nks; ++ks) {
      if (lane == 0 && !*vfail) {
        if (!mbar_wait_one(&bfull[ks % nbs], (ks / nbs) & 1, 0, WL) ||
            !mbar_wait_one(&aempty[ks % kAStages], ((ks / kAStages) & 1) ^ 1, 0, WL))
          *s_fail = 1;
      }
      __syncwarp();
      asm volatile("bar.sync %0, %1;" ::"n"(kBarGo), "n"(kGoCount) : "memory");
    }
  } else if (warp == kLoaderWarp) {
    // ---------------- loader: coordinates + B image by bulk copy ----------------
    if (lane == 0) {
      const uint32_t cbytes = coord_bytes(DIR);
      const uint32_t bbytes = 2 * btile;
      int issued = 0;
      for (int ks = 0; ks < nks; ++ks) {
        const int sb = ks % nbs;
        if (*vfail || !mbar_wait_one(&bempty[sb], ((ks / nbs) & 1) ^ 1, 32, WL)) {
          *s_fail = 1;
          break;
        }
        unsigned char *bdst = bring + sb * bst;
        unsigned char *cdst = bdst + 2 * btile;
        const int k0 = ks * kK;
        mbar_arrive_tx(&bfull[sb], cbytes + bbytes);
        bulk_g2s(bdst, reinterpret_cast<const unsigned char *>(a.bimg) + (size_t)ks * bbytes, bbytes,
                 &bfull[sb]);
        if (DIR == 0) {
          bulk_g2s(cdst, a.ys + k0, cbytes, &bfull[sb]);
        } else {
          // the 32 rows' points, then their normals
          bulk_g2s(cdst, a.xr + k0, cbytes / 2, &bfull[sb]);
          bulk_g2s(cdst + cbytes / 2, a.nr + k0, cbytes / 2, &bfull[sb]);
        }
        ++issued;
      }
      // no copy may still be landing when the CTA exits
      for (int ks = issued > nbs ? issued - nbs : 0; ks < issued; ++ks)
        if (!mbar_wait_one(&bfull[ks % nbs], (ks / nbs) & 1)) *s_fail = 1;
    }
  } else if (warp == kMmaWarp) {
    // ---------------- MMA issue ----------------
    const uint32_t idesc = idesc_tf32(a.np);
    for (int ks = 0; ks < nks; ++ks) {
      const int sa = ks % kAStages, sb = ks % nbs;
      const int kc = ks % kChunk;
      if (lane == 0 && !*vfail) {
        // the B stage (normally landed long ago), and at a chunk start the
        // previous chunk folded out of the accumulator
        if (!mbar_wait_one(&bfull[sb], (ks / nbs) & 1, 0, WL) ||
            (kc == 0 && ks > 0 && !mbar_wait_one(chunk_free, ((ks / kChunk) - 1) & 1, 0, WL)))
          *s_fail = 1;
      }
      __syncwarp();
      asm volatile("bar.sync %0, %1;" ::"n"(kBarAReady), "n"(kGoCount) : "memory");
      if (lane == 0 && !*vfail) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t Ahi = smem_u32(smem + sa * 2 * kTileA), Alo = Ahi + kTileA;
        const uint32_t Bhi = smem_u32(bring + sb * bst), Blo = Bhi + btile;
#pragma unroll
        for (int kk = 0; kk < kK / 8; ++kk) {
          const uint32_t ko = kk * 32;  // 8 TF32 = 32 bytes along the swizzled row
          const uint32_t acc0 = (kc > 0 || kk > 0) ? 1u : 0u;
          mma_tf32(tmem_acc, desc_sw128(Alo + ko), desc_sw128(Bhi + ko), idesc, acc0);
          mma_tf32(tmem_acc, desc_sw128(Ahi + ko), desc_sw128(Blo + ko), idesc, 1u);
          mma_tf32(tmem_acc, desc_sw128(Ahi + ko), desc_sw128(Bhi + ko), idesc, 1u);
        }
        mma_commit(&aempty[sa]);
        mma_commit(&bempty[sb]);
        if (kc == kChunk - 1 || ks == nks - 1) mma_commit(chunk_full);
      }
      __syncwarp();
    }
    if (lane == 0) {
      // after a failure, release the accumulator warps once every MMA issued
      // so far has finished; tensor memory is freed only after that point
      if (*vfail) mma_commit(chunk_full);
      mma_commit(mma_done);
      if (!mbar_wait_one(mma_done, 0)) *s_fail = 1;
    }
  } else {
    // ---------------- accumulator warps: fold chunks, then the epilogue ----------------
    const int q = warp & 3;  // tensor-memory lane quarter of this warp
    const int gm = m0 + q * 32 + lane;
    const uint32_t lane_off = (uint32_t)(q * 32) << 16;
    bool ok = true;
    for (int c = 0; c < nchunks; ++c) {
      if (warp == kAccWarp0 && lane == 0) s_aflag[c & 1] = mbar_wait_one(chunk_full, c & 1, 64, WL) ? 1 : 0;
      asm volatile("bar.sync %0, 128;" ::"n"(kBarAcc) : "memory");
      if (!s_aflag[c & 1]) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const bool last = c == nchunks - 1;
      for (int c0 = 0; c0 < a.np; c0 += 32) {
        float v[32];
        tmem_ld32(tmem_acc + lane_off + (uint32_t)c0, v);
        if (c > 0) {
          float u[32];
          tmem_ld32(tmem_sum + lane_off + (uint32_t)c0, u);
#pragma unroll
          for (int k = 0; k < 32; ++k) v[k] += u[k];
        }
        if (!last) {
          tmem_st32(tmem_sum + lane_off + (uint32_t)c0, v);
          continue;
        }
        if (gm < M_total) {
          float *o = a.out + (size_t)gm * a.R;
#pragma unroll
          for (int k = 0; k < 32; ++k)
            if (c0 + k < a.R) o[c0 + k] = a.coef * v[k];
        }
        if (DIR == 1 && a.part) {
#pragma unroll
          for (int k = 0; k < 32; ++k) {
            double d = 0.0;
            if (gm < M_total && c0 + k < a.R)
              d = (double)(a.coef * v[k]) * (double)a.pdot[(size_t)gm * a.R + c0 + k];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
            if (lane == 0 && c0 + k < a.R) s_red[q * a.R + c0 + k] = d;
          }
        }
      }
      if (!last) {
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(chunk_free);
      }
    }
    if (!ok) *s_fail = 1;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (DIR == 1 && a.part && tid < a.R) {
    a.part[(size_t)blockIdx.x * a.R + tid] =
        *s_fail ? 0.0 : s_red[tid] + s_red[a.R + tid] + s_red[2 * a.R + tid] + s_red[3 * a.R + tid];
  }
  if (tid == 0 && *s_fail && a.err) atomicExch(a.err, 1);
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_acc), "r"(tcols) : "memory");
  }
}

}  // namespace tc
}  // namespace mbc
