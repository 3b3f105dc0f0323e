// FP64-accurate point-kernel matvec on the INT8 tensor cores (tcgen05
// kind::i8) by exact integer slicing of both operands.
//
//   rows:    W[i, r] = coef sum_j G(x_i, n_i, y_j) V[j, r]   (M = rows,    K = sources)
//   columns: T[j, r] = coef sum_i G(x_i, n_i, y_j) W[i, r]   (M = sources, K = rows)
//
// Splitting scheme (Ozaki et al., "Error-free transformations of matrix
// multiplication by using fast routines of matrix multiplication and its
// applications", Numer. Algorithms 59 (2012), with power-of-two scales and
// 8-bit signed digits):
//   * K is cut into chunks of kChunk = 2048 positions.  Every operand value is
//     scaled by a power of two 2^-a per (output row, chunk) for G and per
//     (column, chunk) for the vector block, where 2^a is the smallest power of
//     two >= the largest magnitude in that row / column of the chunk, and
//     rounded to an integer T = rint(v 2^(kW - a)), |T| <= 2^kW, kW = 38.
//   * T is written exactly as kDigits = 5 balanced base-256 digits
//     T = sum_p d_p 256^(4 - p), d_p in [-128, 127]: the bytes of
//     (T + B) xor B with B = 0x8080808080 (each byte u stands for u - 128).
//   * Products of digit planes p (of G) and q (of the vector) with
//     p + q <= 4 (0-based) are formed on the tensor cores and summed exactly
//     in INT32, one accumulator per level l = p + q (|sum| <= 5 * 2048 * 2^14
//     < 2^31; |T| <= 2^38 keeps the top digit in [-64, 64]).  Per product
//     term, rounding T costs at most 2^-38 and the dropped levels l >= 5
//     ~2^-36 of 2^(a+b) <= 4 max|g| max|v| of the chunk, so an output is off
//     by at most 2^-33 sum_c kc max|G_c| max|V_c| (coherent worst case; on
//     MFS operators ~2e-10 relative).
//   * After each chunk the five level accumulators are combined exactly in
//     int64 (Horner in base 256, < 2^58) and added in FP64 with the weight
//     2^(a_row + b_col - kScaleShift).
// Measured in emulation on the normal equations of an MFS scene: operator
// error 1.6e-10 relative at the solution, and PCG with this operator in both
// directions reaches the FP64 true residual of 1e-8 (after one restart from
// the recomputed residual) in 4 % more iterations than the FP64 operator.
//
// G is evaluated with PointKernel<double>::eval, the function the FP64
// CUDA-core kernels use, so the digits encode the same FP64 values.  G does
// not change while a solver lives, so its digit planes are built once per
// solver and direction (oz_digits_kernel: 5 bytes per matrix entry, stored
// in the shared-memory image the MMA reads); a matvec packs only the vector
// block (oz_pack_b_kernel) and runs oz_mma_kernel:
//   one CTA owns 128 outputs x np columns (np <= 96, so the five level
//   accumulators fit 480 tensor-memory columns); adjacent CTAs take the other
//   column groups of the same 128 outputs, so the A planes they share come
//   from L2.  The vector's digit planes are stacked along N in one B image
//   [plane 0 | plane 1 | ... | plane 4] (np rows each), so one MMA of A plane p
//   against the first np (5 - p) rows of B updates the levels p .. 4 at once
//   (tensor-memory columns l np .. ): 8 MMAs per 32-byte k-substep instead
//   of 15.
//     loader warp  -- bulk-copies the B image of a k-step (ring of 2) and the
//                     five A plane tiles (ring of 6 single planes);
//     MMA warp     -- per k-step and plane: waits the tiles, issues the
//                     MMAs (kind::i8, K = 32, N <= 256 per instruction),
//                     commits the A slot; then the B slot; at a chunk end
//                     "chunk_full";
//     8 accumulator warps -- two per tensor-memory lane quarter, half of the
//                     columns each: fold a finished chunk into FP64 sums held
//                     in registers, arrive "chunk_free"; after the last chunk
//                     scale by coef, store, and in the columns direction form
//                     the PCG curvature partials p.t per row tile.
// Every mbarrier wait is bounded, with the failure protocol of the TF32
// tensor-core kernel (record in *err, release the waiters, wait for own
// copies, free tensor memory, return).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "matvec.cuh"
#include "matvec_tc.cuh"

namespace mbc {
namespace oz {

constexpr int kM = 128;                // outputs per CTA (MMA M)
constexpr int kKS = 128;               // K positions per k-step: one 128-byte swizzle row of int8
constexpr int kDigits = 5;             // base-256 digits per value
constexpr int kLevels = kDigits;       // digit-pair levels kept (p + q <= kDigits - 1, 0-based)
constexpr int kW = 8 * kDigits - 2;    // |T| <= 2^kW
constexpr int kChunkSteps = 16;        // k-steps per scale chunk and fold
constexpr int kChunk = kChunkSteps * kKS;
constexpr int kNpMax = 96;             // columns per CTA: kLevels * np <= 480 tensor-memory columns
constexpr int kPlaneBytes = kM * kKS;  // one A digit plane of a k-step: 16 KB
constexpr int kASlots = 6;             // ring of single A planes
constexpr int kBSlots = 2;             // ring of B images
constexpr int kLoaderWarp = 0;
constexpr int kMmaWarp = 1;
constexpr int kAccWarp0 = 2;
constexpr int kAccWarps = 8;
constexpr int kThreads = (kAccWarp0 + kAccWarps) * 32;
constexpr int kBarAcc = 1;             // named barrier of the accumulator warps, once per chunk
constexpr int kScaleShift = 8 * kDigits + 4;  // chunk value = comb 2^(a + b - kScaleShift)
constexpr uint64_t kBias = 0x8080808080ull;   // 128 in each of the kDigits bytes
constexpr uint32_t kWaitLimit = tc::kWaitLimit;
constexpr int kSmemLimit = tc::kSmemLimit;
static_assert(kDigits == 5, "kBias and the level fold are written for five digits");
static_assert(kLevels * kNpMax <= 512, "level accumulators exceed tensor memory");

__host__ __device__ constexpr int bstage_bytes(int np) { return kDigits * np * kKS; }
__host__ __device__ constexpr int tail_bytes(int np) { return 256 + 4 * np * 8; }
__host__ __device__ constexpr int smem_bytes(int np)
{
  return kASlots * kPlaneBytes + kBSlots * bstage_bytes(np) + tail_bytes(np);
}
__host__ __device__ constexpr int tmem_cols_for(int np)
{
  return kLevels * np <= 32 ? 32 : kLevels * np <= 64 ? 64 : kLevels * np <= 128 ? 128
         : kLevels * np <= 256 ? 256 : 512;
}
static_assert(smem_bytes(kNpMax) <= kSmemLimit, "shared memory");

// column groups and padded columns per CTA for R right-hand sides
__host__ __device__ inline int groups_for(int R) { return (R + kNpMax - 1) / kNpMax; }
__host__ __device__ inline int np_for(int R)
{
  const int g = groups_for(R);
  return ((R + g - 1) / g + 15) / 16 * 16;
}

// Sizes and offsets of the device buffers, shared by the kernels, the
// solver's allocations and the host-side layout check.
__host__ __device__ inline int nks_for(int K) { return (K + kKS - 1) / kKS; }
__host__ __device__ inline int nchunks_for(int K) { return (nks_for(K) + kChunkSteps - 1) / kChunkSteps; }
__host__ __device__ inline int row_tiles(int M) { return (M + kM - 1) / kM; }
// A digit planes: [row tile][k-step][digit] tiles of kPlaneBytes
__host__ __device__ inline size_t adig_bytes(int M, int K)
{
  return (size_t)row_tiles(M) * nks_for(K) * kDigits * kPlaneBytes;
}
__host__ __device__ inline size_t adig_offset(int rt, int ks, int p, int nks)
{
  return (((size_t)rt * nks + ks) * kDigits + p) * kPlaneBytes;
}
// A exponents: [row tile][chunk][row]
__host__ __device__ inline size_t aexp_count(int M, int K) { return (size_t)row_tiles(M) * nchunks_for(K) * kM; }
__host__ __device__ inline size_t aexp_index(int rt, int c, int row, int nchunks)
{
  return ((size_t)rt * nchunks + c) * kM + row;
}
// B image: [group][k-step] stages of bstage_bytes(np)
__host__ __device__ inline size_t bimg_bytes(int K, int R)
{
  return (size_t)groups_for(R) * nks_for(K) * bstage_bytes(np_for(R));
}
__host__ __device__ inline size_t bimg_offset(int grp, int ks, int nks, int np)
{
  return ((size_t)grp * nks + ks) * bstage_bytes(np);
}
// B exponents: [group][chunk][column]
__host__ __device__ inline size_t bexp_count(int K, int R)
{
  return (size_t)groups_for(R) * nchunks_for(K) * np_for(R);
}
__host__ __device__ inline size_t bexp_index(int grp, int c, int col, int nchunks, int np)
{
  return ((size_t)grp * nchunks + c) * np + col;
}

// byte offset of the 16-byte group c16 of row `row` in a K-major tile of
// 128-byte rows with the 128-byte swizzle (8-row groups of 1024 bytes)
__host__ __device__ __forceinline__ uint32_t sw128_i8(int row, int c16)
{
  return (uint32_t)((row >> 3) * 1024 + (row & 7) * 128 + (((c16 ^ row) & 7) << 4));
}

// smallest a with m <= 2^a (m >= 0 finite); 0 for m == 0
__device__ __forceinline__ int ceil_exp2(double m)
{
  const unsigned long long b = (unsigned long long)__double_as_longlong(m);
  const int E = (int)((b >> 52) & 0x7FF);
  if (E == 0) return b == 0 ? 0 : -1022;
  return E - 1023 + ((b & 0xFFFFFFFFFFFFFull) != 0 ? 1 : 0);
}

// exponent that marks a column chunk holding a non-finite value: its fold
// weight is infinite, so the outputs it reaches are non-finite
constexpr int kNonFinite = 4096;

// 2^e as a double: 0 below the normal range, infinity above it
__device__ __forceinline__ double pow2(int e)
{
  if (e < -1022) return 0.0;
  if (e > 1023) return __longlong_as_double(0x7FF0000000000000ll);
  return __longlong_as_double((long long)(e + 1023) << 52);
}

// the five digit bytes of T = rint(v 2^(kW - a)) (|v| <= 2^a), as the low
// 40 bits; the two power-of-two scalings are exact
__device__ __forceinline__ uint64_t digit_bytes(double v, int a)
{
  const long long T = __double2ll_rn((v * pow2(-a)) * pow2(kW));
  return ((uint64_t)(T + (long long)kBias)) ^ kBias;
}

// ---------------------------------------------------------------------------
// Digit-kernel modes: exponents (pass 1: the row maxima, written to aexp),
// digits (pass 2: the planes, with the exponents of pass 1 or, alone, read
// back from aexp), or both.  When the planes of every row do not fit in
// device memory, the exponents are computed once and the planes are rebuilt
// slab by slab (rows [rt0, rt0 + gridDim.y) tiles) for every matvec.
constexpr int kModeExps = 1;
constexpr int kModeDigits = 2;

// ---------------------------------------------------------------------------
// A digit planes of G for one direction.  Grid (chunks, row tiles of the
// slab), 256 threads; global row tile = rt0 + blockIdx.y, plane tile index =
// blockIdx.y (the slab's own buffer).  Layout: adig[((rt * nks + ks) * kDigits + p) * kPlaneBytes + ...]
// with the swizzled tile image; aexp[(rt * nchunks + c) * kM + row].  Rows or
// K positions past the ends get digit 0.  A non-finite G (coincident point
// and source) sets *err = 3 and counts as 0.
// Shared memory: kChunk float4 (DIR 0: sources) or 2 kChunk (DIR 1: points,
// normals).
template <int DIR>
__global__ void __launch_bounds__(256) oz_digits_kernel(const float4 *__restrict__ xr,
                                                        const float4 *__restrict__ nr,
                                                        const float4 *__restrict__ ys, int nf, int n,
                                                        int8_t *__restrict__ adig, size_t adig_size,
                                                        int32_t *__restrict__ aexp, size_t aexp_size,
                                                        int rt0, int mode, const int32_t *__restrict__ done,
                                                        int32_t *__restrict__ err)
{
  if (done && *done) return;  // a slab rebuild after the PCG stopped
  extern __shared__ float4 sco[];
  const int M = DIR == 0 ? nf : n;
  const int K = DIR == 0 ? n : nf;
  const int c = blockIdx.x, rt = rt0 + (int)blockIdx.y, rt_local = (int)blockIdx.y;
  const int nks = nks_for(K);
  const int nchunks = nchunks_for(K);
  const int ks0 = c * kChunkSteps;
  const int ks1 = min(ks0 + kChunkSteps, nks);
  const int kbase = ks0 * kKS;
  const int kcount = min(kChunk, K - kbase);
  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int t = threadIdx.x; t < kChunk; t += blockDim.x) {
    if (DIR == 0) {
      sco[t] = t < kcount ? ys[kbase + t] : zero;
    } else {
      sco[t] = t < kcount ? xr[kbase + t] : zero;
      sco[kChunk + t] = t < kcount ? nr[kbase + t] : zero;
    }
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane >> 3, c16 = lane & 7;  // row of the warp's four, 16-byte group of the row
  float4 own[4], own_n[4];
  bool valid[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int gm = rt * kM + 32 * u + 4 * warp + sub;
    valid[u] = gm < M;
    own[u] = own_n[u] = zero;
    if (valid[u]) {
      if (DIR == 0) {
        own[u] = xr[gm];
        own_n[u] = nr[gm];
      } else {
        own[u] = ys[gm];
      }
    }
  }
  auto eval = [&](int u, int k) -> double {
    return DIR == 0 ? PointKernel<double>::eval(own[u], own_n[u], sco[k])
                    : PointKernel<double>::eval(sco[k], sco[kChunk + k], own[u]);
  };
  // pass 1: the largest |G| of each row over the chunk
  double mx[4] = {0.0, 0.0, 0.0, 0.0};
  bool bad = false;
  for (int ks = ks0; ks < ((mode & kModeExps) ? ks1 : ks0); ++ks) {
    const int kk0 = (ks - ks0) * kKS + c16 * 16;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (!valid[u]) continue;
      for (int e = 0; e < 16; ++e) {
        const int k = kk0 + e;
        if (k >= kcount) break;
        const double g = eval(u, k);
        if (isfinite(g)) mx[u] = fmax(mx[u], fabs(g));
        else bad = true;
      }
    }
  }
  if (bad) atomicMax(err, 3);
  int ea[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const size_t ei = aexp_index(rt, c, 32 * u + 4 * warp + sub, nchunks);
    if (mode & kModeExps) {
#pragma unroll
      for (int o = 1; o < 8; o <<= 1) mx[u] = fmax(mx[u], __shfl_xor_sync(0xffffffffu, mx[u], o));
      ea[u] = ceil_exp2(mx[u]);
      if (c16 == 0) {
        if (ei < aexp_size) aexp[ei] = ea[u];
        else atomicMax(err, 4);
      }
    } else {
      ea[u] = 0;
      if (ei < aexp_size) ea[u] = aexp[ei];
      else atomicMax(err, 4);
    }
  }
  if (!(mode & kModeDigits)) return;
  // pass 2: digits, one 16-byte group of five planes per (row, c16)
  for (int ks = ks0; ks < ks1; ++ks) {
    const int kk0 = (ks - ks0) * kKS + c16 * 16;
    const size_t tile_off = adig_offset(rt_local, ks, 0, nks);
    unsigned char *tile = reinterpret_cast<unsigned char *>(adig) + tile_off;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int row = 32 * u + 4 * warp + sub;
      uint32_t w[kDigits][4];
#pragma unroll
      for (int p = 0; p < kDigits; ++p) w[p][0] = w[p][1] = w[p][2] = w[p][3] = 0u;
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const int k = kk0 + e;
        uint64_t tb = 0;
        if (valid[u] && k < kcount) {
          const double g = eval(u, k);
          if (isfinite(g)) tb = digit_bytes(g, ea[u]);
        }
#pragma unroll
        for (int p = 0; p < kDigits; ++p)
          w[p][e >> 2] |= (uint32_t)((tb >> (8 * (kDigits - 1 - p))) & 0xFFu) << (8 * (e & 3));
      }
      const uint32_t off = sw128_i8(row, c16);
      if (tile_off + (size_t)(kDigits - 1) * kPlaneBytes + off + 16 > adig_size) {
        atomicMax(err, 4);  // outside the planes: skip the stores
        continue;
      }
#pragma unroll
      for (int p = 0; p < kDigits; ++p)
        *reinterpret_cast<uint4 *>(tile + (size_t)p * kPlaneBytes + off) = make_uint4(w[p][0], w[p][1], w[p][2], w[p][3]);
    }
  }
}

// ---------------------------------------------------------------------------
// B image of the input block vin (K x R, row-major FP64) for one matvec.
// Grid (chunks, groups), 512 threads.  Layout: bimg[(grp * nks + ks) *
// bstage_bytes(np) + ...], rows p * np + r (plane p, column grp * np + r) of
// the swizzled image; bexp[(grp * nchunks + c) * np + r].
__global__ void __launch_bounds__(512) oz_pack_b_kernel(const double *__restrict__ vin, int K, int R,
                                                        int np, int8_t *__restrict__ bimg, size_t bimg_size,
                                                        int32_t *__restrict__ bexp, size_t bexp_size,
                                                        const int32_t *__restrict__ done,
                                                        int32_t *__restrict__ err)
{
  if (done && *done) return;
  __shared__ double s_max[16][kNpMax];
  __shared__ int s_exp[kNpMax];
  const int c = blockIdx.x, grp = blockIdx.y;
  const int nks = nks_for(K);
  const int nchunks = nchunks_for(K);
  const int ks0 = c * kChunkSteps;
  const int ks1 = min(ks0 + kChunkSteps, nks);
  const int kbase = ks0 * kKS;
  const int kcount = min(kChunk, K - kbase);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // pass 1: column maxima over the chunk (warp w takes rows w, w + 16, ...)
  for (int cb = 0; cb < np; cb += 32) {
    const int col = cb + lane;
    const int gc = grp * np + col;
    double m = 0.0;
    bool finite = true;
    if (col < np && gc < R)
      for (int k = warp; k < kcount; k += 16) {
        const double x = vin[(size_t)(kbase + k) * R + gc];
        finite = finite && isfinite(x);
        m = fmax(m, fabs(x));
      }
    if (col < np) s_max[warp][col] = finite ? m : __longlong_as_double(0x7FF0000000000000ll);
  }
  __syncthreads();
  for (int col = threadIdx.x; col < np; col += blockDim.x) {
    double m = 0.0;
#pragma unroll
    for (int w = 0; w < 16; ++w) m = fmax(m, s_max[w][col]);
    const int e = isfinite(m) ? ceil_exp2(m) : kNonFinite;
    s_exp[col] = e;
    const size_t ei = bexp_index(grp, c, col, nchunks, np);
    if (ei < bexp_size) bexp[ei] = e;
    else atomicMax(err, 4);
  }
  __syncthreads();
  // pass 2: units (k-step, column, 16-byte group); lanes run over columns
  const int units = (ks1 - ks0) * np * 8;
  for (int t = threadIdx.x; t < units; t += blockDim.x) {
    const int col = t % np;
    const int rest = t / np;
    const int c16 = rest & 7;
    const int ks = ks0 + (rest >> 3);
    const int gc = grp * np + col;
    const int kk0 = (ks - ks0) * kKS + c16 * 16;
    uint32_t w[kDigits][4];
#pragma unroll
    for (int p = 0; p < kDigits; ++p) w[p][0] = w[p][1] = w[p][2] = w[p][3] = 0u;
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      const int k = kk0 + e;
      uint64_t tb = 0;
      if (gc < R && k < kcount) tb = digit_bytes(vin[(size_t)(kbase + k) * R + gc], s_exp[col]);
#pragma unroll
      for (int p = 0; p < kDigits; ++p)
        w[p][e >> 2] |= (uint32_t)((tb >> (8 * (kDigits - 1 - p))) & 0xFFu) << (8 * (e & 3));
    }
    const size_t img_off = bimg_offset(grp, ks, nks, np);
    unsigned char *img = reinterpret_cast<unsigned char *>(bimg) + img_off;
    if (img_off + sw128_i8((kDigits - 1) * np + col, c16) + 16 > bimg_size) {
      atomicMax(err, 4);  // outside the image: skip the stores
      continue;
    }
#pragma unroll
    for (int p = 0; p < kDigits; ++p)
      *reinterpret_cast<uint4 *>(img + sw128_i8(p * np + col, c16)) = make_uint4(w[p][0], w[p][1], w[p][2], w[p][3]);
  }
}

// ---------------------------------------------------------------------------
// The MMA kernel.

// kind::i8, S32 accumulate, A and B signed 8-bit, K-major, M = 128, N = nn
__host__ __device__ __forceinline__ constexpr uint32_t idesc_i8(int nn)
{
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(nn >> 3) << 17) | ((uint32_t)(kM >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                       uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

// the five level accumulators of 8 columns of this warp's lanes: addresses
// t0 + l * stride, one wait for all loads inside the same statement
__device__ __forceinline__ void tmem_ld_levels8(uint32_t t0, uint32_t stride, int32_t (&v)[kLevels][8])
{
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%40];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%8,%9,%10,%11,%12,%13,%14,%15}, [%41];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%16,%17,%18,%19,%20,%21,%22,%23}, [%42];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%24,%25,%26,%27,%28,%29,%30,%31}, [%43];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%32,%33,%34,%35,%36,%37,%38,%39}, [%44];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(v[0][0]), "=r"(v[0][1]), "=r"(v[0][2]), "=r"(v[0][3]), "=r"(v[0][4]), "=r"(v[0][5]),
        "=r"(v[0][6]), "=r"(v[0][7]), "=r"(v[1][0]), "=r"(v[1][1]), "=r"(v[1][2]), "=r"(v[1][3]),
        "=r"(v[1][4]), "=r"(v[1][5]), "=r"(v[1][6]), "=r"(v[1][7]), "=r"(v[2][0]), "=r"(v[2][1]),
        "=r"(v[2][2]), "=r"(v[2][3]), "=r"(v[2][4]), "=r"(v[2][5]), "=r"(v[2][6]), "=r"(v[2][7]),
        "=r"(v[3][0]), "=r"(v[3][1]), "=r"(v[3][2]), "=r"(v[3][3]), "=r"(v[3][4]), "=r"(v[3][5]),
        "=r"(v[3][6]), "=r"(v[3][7]), "=r"(v[4][0]), "=r"(v[4][1]), "=r"(v[4][2]), "=r"(v[4][3]),
        "=r"(v[4][4]), "=r"(v[4][5]), "=r"(v[4][6]), "=r"(v[4][7])
      : "r"(t0), "r"(t0 + stride), "r"(t0 + 2 * stride), "r"(t0 + 3 * stride), "r"(t0 + 4 * stride)
      : "memory");
}

struct OzArgs {
  const int8_t *adig;   // A digit planes of this direction
  const int32_t *aexp;  // A exponents [row tile][chunk][128]
  const int8_t *bimg;   // B image of the input block
  const int32_t *bexp;  // B exponents [group][chunk][np]
  size_t adig_size, bimg_size;  // bytes
  size_t aexp_size, bexp_size;  // entries
  int rt0;              // first row tile of this launch (slab); adig holds the slab's planes
  double *out;          // M x R
  int M, K, R, groups;  // outputs, reduction length, columns, column groups
  double coef;
  const double *pdot;   // columns: p (M x R) for the curvature partials, or NULL
  double *part;         // columns: per-row-tile partials (row tiles x R)
  const int32_t *done;  // PCG all-stopped flag (may be NULL)
  int32_t *err;         // the largest code raised (atomicMax): 1 a bounded wait expired, 2 shared
                        // memory misaligned, 4 an index outside its buffer (access skipped)
  // polls after which a wait for a partner gives up (0: kWaitLimit); the
  // waits that drain the CTA's own copies and MMAs always use kWaitLimit
  uint32_t wait_limit;
};

// NPH = np / 2 columns per accumulator warp
template <int NPH>
__global__ void __launch_bounds__(kThreads, 1) oz_mma_kernel(OzArgs a)
{
  if (a.done && *a.done) return;
  constexpr int NP = 2 * NPH;
  constexpr int BST = bstage_bytes(NP);
  constexpr int TCOLS = tmem_cols_for(NP);
  static_assert(NPH % 8 == 0 && NP <= kNpMax, "columns per CTA");
  extern __shared__ __align__(1024) unsigned char smem[];
  if (tc::smem_u32(smem) & 1023u) {
    if (threadIdx.x == 0) atomicMax(a.err, 2);
    return;
  }
  unsigned char *aring = smem;
  unsigned char *bring = smem + kASlots * kPlaneBytes;
  unsigned char *tail = bring + kBSlots * BST;
  uint64_t *afull = reinterpret_cast<uint64_t *>(tail);  // A slot landed
  uint64_t *aempty = afull + kASlots;                    // A slot read by its MMAs
  uint64_t *bfull = aempty + kASlots;                    // B slot landed
  uint64_t *bempty = bfull + kBSlots;                    // B slot read by its MMAs
  uint64_t *chunk_full = bempty + kBSlots;
  uint64_t *chunk_free = chunk_full + 1;
  uint64_t *mma_done = chunk_free + 1;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mma_done + 1);
  int *s_fail = reinterpret_cast<int *>(tmem_slot + 1);
  volatile int *s_aflag = s_fail + 1;                   // [2]
  double *s_red = reinterpret_cast<double *>(tail + 256);  // [4][NP]

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int rt_local = blockIdx.x / a.groups, grp = blockIdx.x - rt_local * a.groups;
  const int rt = a.rt0 + rt_local;  // global row tile: exponents, outputs, partials
  const int m0 = rt * kM;
  const int nks = nks_for(a.K);
  const int nchunks = nchunks_for(a.K);
  // the partner-wait limit, read from the parameter bank at each use
#define WL (a.wait_limit ? a.wait_limit : kWaitLimit)

  if (tid == 0) {
    for (int s = 0; s < kASlots; ++s) {
      tc::mbar_init(&afull[s], 1);
      tc::mbar_init(&aempty[s], 1);
    }
    for (int s = 0; s < kBSlots; ++s) {
      tc::mbar_init(&bfull[s], 1);
      tc::mbar_init(&bempty[s], 1);
    }
    tc::mbar_init(chunk_full, 1);
    tc::mbar_init(chunk_free, kAccWarps);
    tc::mbar_init(mma_done, 1);
    *s_fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     tc::smem_u32(tmem_slot)),
                 "r"(TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  volatile int *vfail = s_fail;

  if (warp == kLoaderWarp) {
    // ---------------- loader: B image per k-step, then its five A planes ----------------
    if (lane == 0) {
      const unsigned char *abase = reinterpret_cast<const unsigned char *>(a.adig);
      const unsigned char *bbase = reinterpret_cast<const unsigned char *>(a.bimg);
      int b_issued = 0, a_issued = 0;
      for (int ks = 0; ks < nks; ++ks) {
        const int sb = ks % kBSlots;
        if (*vfail || !tc::mbar_wait_one(&bempty[sb], ((ks / kBSlots) & 1) ^ 1, 32, WL)) {
          *s_fail = 1;
          break;
        }
        const size_t boff = bimg_offset(grp, ks, nks, NP);
        if (boff + BST > a.bimg_size) {
          atomicMax(a.err, 4);  // outside the image: no copy, fail
          *s_fail = 1;
          break;
        }
        tc::mbar_arrive_tx(&bfull[sb], BST);
        tc::bulk_g2s(bring + sb * BST, bbase + boff, BST, &bfull[sb]);
        ++b_issued;
        bool ok = true;
        for (int p = 0; p < kDigits; ++p) {
          const int t = ks * kDigits + p, sa = t % kASlots;
          const size_t aoff = adig_offset(rt_local, ks, p, nks);
          if (aoff + kPlaneBytes > a.adig_size) {
            atomicMax(a.err, 4);  // outside the planes: no copy, fail
            ok = false;
            break;
          }
          if (!tc::mbar_wait_one(&aempty[sa], ((t / kASlots) & 1) ^ 1, 32, WL)) {
            ok = false;
            break;
          }
          tc::mbar_arrive_tx(&afull[sa], kPlaneBytes);
          tc::bulk_g2s(aring + sa * kPlaneBytes, abase + aoff, kPlaneBytes, &afull[sa]);
          ++a_issued;
        }
        if (!ok) {
          *s_fail = 1;
          break;
        }
      }
      // no copy may still be landing when the CTA exits
      for (int ks = b_issued > kBSlots ? b_issued - kBSlots : 0; ks < b_issued; ++ks)
        if (!tc::mbar_wait_one(&bfull[ks % kBSlots], (ks / kBSlots) & 1)) *s_fail = 1;
      for (int t = a_issued > kASlots ? a_issued - kASlots : 0; t < a_issued; ++t)
        if (!tc::mbar_wait_one(&afull[t % kASlots], (t / kASlots) & 1)) *s_fail = 1;
    }
  } else if (warp == kMmaWarp) {
    // ---------------- MMA issue ----------------
    if (lane == 0) {
      for (int ks = 0; ks < nks; ++ks) {
        const int kc = ks % kChunkSteps, sb = ks % kBSlots;
        // the B image, and at a chunk start the previous chunk folded out
        if (*vfail || !tc::mbar_wait_one(&bfull[sb], (ks / kBSlots) & 1, 0, WL) ||
            (kc == 0 && ks > 0 && !tc::mbar_wait_one(chunk_free, ((ks / kChunkSteps) - 1) & 1, 32, WL))) {
          *s_fail = 1;
          break;
        }
        const uint32_t B0 = tc::smem_u32(bring + sb * BST);
        bool ok = true;
        for (int p = 0; p < kDigits; ++p) {
          const int t = ks * kDigits + p, sa = t % kASlots;
          if (!tc::mbar_wait_one(&afull[sa], (t / kASlots) & 1, 0, WL)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t A0 = tc::smem_u32(aring + sa * kPlaneBytes);
          const int nt = NP * (kDigits - p);  // B rows of planes 0 .. kDigits-1-p
#pragma unroll
          for (int kk = 0; kk < kKS / 32; ++kk) {
            // the first MMAs of a chunk (plane 0 covers every level column) start from zero
            const uint32_t acc = (kc == 0 && p == 0 && kk == 0) ? 0u : 1u;
            for (int n0 = 0; n0 < nt; n0 += 256) {
              const int nn = nt - n0 < 256 ? nt - n0 : 256;
              mma_i8(tmem + (uint32_t)(p * NP + n0), tc::desc_sw128(A0 + kk * 32),
                     tc::desc_sw128(B0 + (uint32_t)(n0 / 8) * 1024 + kk * 32), idesc_i8(nn), acc);
            }
          }
          tc::mma_commit(&aempty[sa]);
        }
        if (!ok) {
          *s_fail = 1;
          break;
        }
        tc::mma_commit(&bempty[sb]);
        if (kc == kChunkSteps - 1 || ks == nks - 1) tc::mma_commit(chunk_full);
      }
      // after a failure, release the accumulator warps once every MMA issued
      // so far has finished; tensor memory is freed only after that point
      if (*vfail) tc::mma_commit(chunk_full);
      tc::mma_commit(mma_done);
      if (!tc::mbar_wait_one(mma_done, 0)) *s_fail = 1;
    }
  } else {
    // ---------------- accumulator warps: fold chunks, then the epilogue ----------------
    const int aw = warp - kAccWarp0;  // 0 .. 7
    const int qd = warp & 3;          // tensor-memory lane quarter of this warp
    const int c0 = (aw >> 2) * NPH;   // first column of this warp
    const int row = qd * 32 + lane;
    const int gm = m0 + row;
    const uint32_t lane_off = (uint32_t)(qd * 32) << 16;
    double sum[NPH];
#pragma unroll
    for (int k = 0; k < NPH; ++k) sum[k] = 0.0;
    bool ok = true;
    for (int c = 0; c < nchunks; ++c) {
      if (aw == 0 && lane == 0) s_aflag[c & 1] = tc::mbar_wait_one(chunk_full, c & 1, 64, WL) ? 1 : 0;
      asm volatile("bar.sync %0, %1;" ::"n"(kBarAcc), "n"(kAccWarps * 32) : "memory");
      if (!s_aflag[c & 1]) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      // the check covers the whole CTA's exponents, so every accumulator
      // thread takes the same branch (a partial exit would strand the others
      // at the named barrier)
      if (aexp_index(rt, c, kM - 1, nchunks) >= a.aexp_size ||
          bexp_index(grp, c, 0, nchunks, NP) + NP > a.bexp_size) {
        if (aw == 0 && lane == 0) atomicMax(a.err, 4);  // no fold, fail (the MMA warp's wait expires)
        ok = false;
        break;
      }
      const int ea = a.aexp[aexp_index(rt, c, row, nchunks)];
      const int32_t *eb = a.bexp + bexp_index(grp, c, c0, nchunks, NP);
#pragma unroll
      for (int g = 0; g < NPH / 8; ++g) {
        int32_t v[kLevels][8];
        tmem_ld_levels8(tmem + lane_off + (uint32_t)(c0 + g * 8), (uint32_t)NP, v);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          long long comb = v[0][k];
#pragma unroll
          for (int l = 1; l < kLevels; ++l) comb = comb * 256 + v[l][k];
          sum[g * 8 + k] = fma((double)comb, pow2(ea + eb[g * 8 + k] - kScaleShift), sum[g * 8 + k]);
        }
      }
      if (c < nchunks - 1) {
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(chunk_free);
      }
    }
    if (!ok) *s_fail = 1;
    const int col0 = grp * NP + c0;
    if (ok && gm < a.M) {
      double *o = a.out + (size_t)gm * a.R + col0;
#pragma unroll
      for (int k = 0; k < NPH; ++k)
        if (col0 + k < a.R) o[k] = a.coef * sum[k];
    }
    if (a.part) {
#pragma unroll
      for (int k = 0; k < NPH; ++k) {
        double d = 0.0;
        if (gm < a.M && col0 + k < a.R) d = a.coef * sum[k] * a.pdot[(size_t)gm * a.R + col0 + k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
        if (lane == 0) s_red[qd * NP + c0 + k] = d;
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (a.part && tid < NP && grp * NP + tid < a.R) {
    a.part[(size_t)rt * a.R + grp * NP + tid] =
        *s_fail ? 0.0 : s_red[tid] + s_red[NP + tid] + s_red[2 * NP + tid] + s_red[3 * NP + tid];
  }
  if (tid == 0 && *s_fail && a.err) atomicMax(a.err, 1);
  if (warp == 0) {
    // warp 0 is also the loader, whose lane 0 ran alone: reconverge before
    // the warp-wide (.sync.aligned) dealloc
    __syncwarp();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS) : "memory");
  }
}

#undef WL

}  // namespace oz
}  // namespace mbc
