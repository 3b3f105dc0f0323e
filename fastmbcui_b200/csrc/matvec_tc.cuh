// Tensor-core (tcgen05) form of the batched point-kernel matvec.
//
//   rows:    W[i, r] = coef sum_j G(x_i, n_i, y_j) V[j, r]   (M = rows,    K = sources)
//   columns: T[j, r] = coef sum_i G(x_i, n_i, y_j) W[i, r]   (M = sources, K = rows)
//
// G = ((x - y).n) / |x - y|^3 is generated by SIMT warps tile by tile and
// never stored.  One CTA owns 128 outputs (the MMA M) and all R columns (the
// MMA N, R padded to a multiple of 16, at most 256); its accumulator lives in
// tensor memory.  Per k-step of 32:
//   * 8 producer warps evaluate the 128 x 32 tile of G in FP32, split each
//     value into TF32 hi + lo (hi = rna(v), lo = rna(v - hi)), and stage the
//     vector block (R x 32) the same way; both are stored K-major with the
//     128-byte swizzle the MMA descriptors expect;
//   * one thread issues 4 x 3 tcgen05.mma.kind::tf32 (K = 8 each):
//     hi*hi + hi*lo + lo*hi ("3xTF32"), which keeps FP32-level accuracy;
//   * a 2-stage ring of mbarriers (full: producers -> MMA, empty: MMA commit
//     -> producers) overlaps generation with the tensor pipe.
// The epilogue drains TMEM with tcgen05.ld (warps 0-3, one lane quarter
// each), scales by coef and stores; the columns direction also forms the PCG
// curvature partials p.t per CTA.
//
// Every mbarrier wait is bounded: on expiry the kernel sets *err, stops
// waiting, still commits its issued MMAs to the final barrier, frees its
// tensor memory and returns.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "matvec.cuh"

namespace mbc {
namespace tc {

constexpr int kM = 128;        // MMA M (outputs per CTA)
constexpr int kK = 32;         // k-step (one 128-byte swizzle row of TF32)
constexpr int kStages = 2;
constexpr int kProducerWarps = 8;
constexpr int kThreads = (kProducerWarps + 1) * 32;  // + the MMA warp
constexpr uint32_t kWaitLimit = 1u << 22;            // polls of a bounded wait

constexpr int kTileA = kM * kK * 4;  // bytes of one A operand tile (16 KB)

__host__ __device__ constexpr int tile_b_bytes(int np) { return np * kK * 4; }
__host__ __device__ constexpr int stage_bytes(int np) { return 2 * kTileA + 2 * tile_b_bytes(np); }
// dynamic shared memory: 1 KB alignment slack + stages + 256 B of barriers
// + the epilogue's per-warp partial sums (4 warps x 256 columns x 8 B)
__host__ __device__ constexpr int smem_bytes(int np) { return 1024 + kStages * stage_bytes(np) + 256 + 8192; }

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
  return (uint32_t)__cvta_generic_to_shared(p);
}

// byte offset of element (row, k) in a K-major, 128B-swizzled tile whose
// rows are 32 TF32 values (128 B); the tile base is 1024-byte aligned
__device__ __forceinline__ uint32_t sw128(int row, int k)
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

// bounded wait for the phase with the given parity; false on expiry
__device__ __forceinline__ bool mbar_wait_one(uint64_t *bar, uint32_t parity)
{
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < kWaitLimit; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// warp-uniform bounded wait: lane 0 polls, the outcome is broadcast and
// __syncwarp orders the other lanes after lane 0's acquire
__device__ __forceinline__ bool mbar_wait_warp(uint64_t *bar, uint32_t parity)
{
  int got = 0;
  if ((threadIdx.x & 31) == 0) got = mbar_wait_one(bar, parity) ? 1 : 0;
  got = __shfl_sync(0xffffffffu, got, 0);
  __syncwarp();
  return got != 0;
}

__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr)
{
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);  // start address
  d |= (uint64_t)1 << 16;                            // LBO (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;                  // SBO: 8 rows x 128 B
  d |= (uint64_t)1 << 46;                            // descriptor version (sm100)
  d |= (uint64_t)2 << 61;                            // SWIZZLE_128B
  return d;
}

// kind::tf32, FP32 accumulate, A and B K-major, M = 128, N = np
__device__ __forceinline__ uint32_t idesc_tf32(int np)
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

struct TcArgs {
  const float4 *xr, *nr;  // collocation rows (original order)
  const float4 *ys;       // sources (new order)
  int nf, n;
  const float *vin;       // rows: V (n x R); columns: W (nf x R)
  float *out;             // rows: W (nf x R); columns: T (n x R)
  int R, np;              // columns and padded MMA N (multiple of 16, <= 256)
  int tmem_cols;          // power of two >= np, >= 32
  float coef;
  const float *pdot;      // columns: p (n x R) for the curvature partials, or NULL
  double *part;           // columns: per-CTA partials (gridDim.x x R)
  const int32_t *done;    // PCG all-stopped flag (may be NULL)
  int32_t *err;           // set to 1 when a bounded wait expires
};

template <int DIR>
__global__ void __launch_bounds__(kThreads, 1) pk_tc_kernel(TcArgs a)
{
  if (a.done && *a.done) return;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  unsigned char *base = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  const int sb = stage_bytes(a.np);
  unsigned char *tail = base + kStages * sb;
  uint64_t *full = reinterpret_cast<uint64_t *>(tail);
  uint64_t *empty = full + kStages;
  uint64_t *done_bar = empty + kStages;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done_bar + 1);
  int *s_fail = reinterpret_cast<int *>(tmem_slot + 1);
  double *s_red = reinterpret_cast<double *>(tail + 256);  // [4][R] warp partials (columns)

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int M_total = DIR == 0 ? a.nf : a.n;
  const int K_total = DIR == 0 ? a.n : a.nf;
  const int m0 = blockIdx.x * kM;
  const int nks = (K_total + kK - 1) / kK;

  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], kProducerWarps);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done_bar, 1);
    *s_fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(a.tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  // B rows np > R stay zero: clear every stage's B tiles once
  for (int s = 0; s < kStages; ++s) {
    uint4 *b = reinterpret_cast<uint4 *>(base + s * sb + 2 * kTileA);
    for (int t = tid; t < 2 * tile_b_bytes(a.np) / 16; t += kThreads) b[t] = make_uint4(0, 0, 0, 0);
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem_d = *tmem_slot;

  if (warp < kProducerWarps) {
    // ---------------- producers ----------------
    const int row = (warp & 3) * 32 + lane;  // A row (output) owned by this thread
    const int khalf = warp >> 2;             // which 16 of the 32 k
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
    bool ok = true;
    for (int ks = 0; ks < nks && ok; ++ks) {
      const int s = ks % kStages;
      if (!mbar_wait_warp(&empty[s], ((ks / kStages) & 1) ^ 1)) {
        ok = false;
        break;
      }
      unsigned char *st = base + s * sb;
      unsigned char *Ahi = st, *Alo = st + kTileA;
      unsigned char *Bhi = st + 2 * kTileA, *Blo = Bhi + tile_b_bytes(a.np);
      const int k0 = ks * kK;
      // A: 16 values of this thread's row
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        uint32_t h[4], l[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int k = khalf * 16 + q * 4 + e;
          const int gk = k0 + k;
          float g = 0.f;
          if (gk < K_total && gm < M_total) {
            if (DIR == 0) g = PointKernel<float>::eval(own, own_n, __ldg(a.ys + gk));
            else g = PointKernel<float>::eval(__ldg(a.xr + gk), __ldg(a.nr + gk), own);
          }
          split_tf32(g, h[e], l[e]);
        }
        const uint32_t off = sw128(row, khalf * 16 + q * 4);
        *reinterpret_cast<uint4 *>(Ahi + off) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4 *>(Alo + off) = make_uint4(l[0], l[1], l[2], l[3]);
      }
      // B: chunks of 4 consecutive k of one column r; element (r, k) = vin[k0 + k][r]
      const int nchunk = a.R * (kK / 4);
      for (int c = tid; c < nchunk; c += kProducerWarps * 32) {
        const int r = c % a.R, kq = c / a.R;
        uint32_t h[4], l[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int gk = k0 + kq * 4 + e;
          const float v = gk < K_total ? __ldg(a.vin + (size_t)gk * a.R + r) : 0.f;
          split_tf32(v, h[e], l[e]);
        }
        const uint32_t off = sw128(r, kq * 4);
        *reinterpret_cast<uint4 *>(Bhi + off) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4 *>(Blo + off) = make_uint4(l[0], l[1], l[2], l[3]);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&full[s]);
    }
    if (!ok) *s_fail = 1;
  } else if (lane == 0) {
    // ---------------- MMA issue ----------------
    const uint32_t idesc = idesc_tf32(a.np);
    for (int ks = 0; ks < nks; ++ks) {
      const int s = ks % kStages;
      if (!mbar_wait_one(&full[s], (ks / kStages) & 1)) {
        *s_fail = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t st = smem_u32(base + s * sb);
      const uint32_t Ahi = st, Alo = st + kTileA;
      const uint32_t Bhi = st + 2 * kTileA, Blo = Bhi + tile_b_bytes(a.np);
#pragma unroll
      for (int kk = 0; kk < kK / 8; ++kk) {
        const uint32_t ko = kk * 32;  // 8 TF32 = 32 bytes along the swizzled row
        const uint32_t acc0 = (ks > 0 || kk > 0) ? 1u : 0u;
        mma_tf32(tmem_d, desc_sw128(Alo + ko), desc_sw128(Bhi + ko), idesc, acc0);
        mma_tf32(tmem_d, desc_sw128(Ahi + ko), desc_sw128(Blo + ko), idesc, 1u);
        mma_tf32(tmem_d, desc_sw128(Ahi + ko), desc_sw128(Bhi + ko), idesc, 1u);
      }
      mma_commit(&empty[s]);
    }
    // completes when every MMA issued above has finished
    mma_commit(done_bar);
  }

  // ---------------- epilogue: warps 0-3 ----------------
  if (warp < 4) {
    const bool have = mbar_wait_warp(done_bar, 0);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!have) *s_fail = 1;
    const int row = warp * 32 + lane;
    const int gm = m0 + row;
    for (int c0 = 0; c0 < a.np; c0 += 32) {
      float v[32];
      tmem_ld32(tmem_d + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (have && gm < M_total) {
        float *o = a.out + (size_t)gm * a.R;
#pragma unroll
        for (int k = 0; k < 32; ++k)
          if (c0 + k < a.R) o[c0 + k] = a.coef * v[k];
      }
      if (DIR == 1 && a.part) {
#pragma unroll
        for (int k = 0; k < 32; ++k) {
          double d = 0.0;
          if (have && gm < M_total && c0 + k < a.R)
            d = (double)(a.coef * v[k]) * (double)a.pdot[(size_t)gm * a.R + c0 + k];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
          if (lane == 0 && c0 + k < a.R) s_red[warp * a.R + c0 + k] = d;
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (DIR == 1 && a.part && tid < a.R) {
    a.part[(size_t)blockIdx.x * a.R + tid] =
        s_red[tid] + s_red[a.R + tid] + s_red[2 * a.R + tid] + s_red[3 * a.R + tid];
  }
  if (tid == 0 && *s_fail && a.err) atomicExch(a.err, 1);
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_d), "r"(a.tmem_cols)
                 : "memory");
  }
}

}  // namespace tc
}  // namespace mbc
