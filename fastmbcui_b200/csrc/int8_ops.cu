// The FP64-accurate INT8 tensor-core matvec inside the solver: dispatch of
// the pack and MMA kernels (matvec_oz.cuh), the digit planes of G (full or
// slab by slab), the first-use check against the FP64 kernels, and the C
// entry points that select and prepare it.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "cuda_util.h"
#include "int8_ops.h"
#include "matvec_oz.cuh"
#include "solver.h"

namespace mbc {

// FP64-accurate INT8 path: an FP64 point-kernel matvec once the digit
// planes of G are built (Solver::ensure_oz)
bool use_oz(const Solver &S)
{
  return S.fp64_matvec == MBC_FP64_MATVEC_INT8 && S.oz_ready && S.op.kind == MBC_OP_POINT_KERNEL;
}

// dst[k, c] = src[idx[k], c] (K x R, FP64): the vector block in the order the
// planes' reduction axis walks
__global__ void oz_gather_kernel(int K, int R, const int32_t *__restrict__ idx, const double *__restrict__ src,
                                 double *__restrict__ dst, const int32_t *__restrict__ done)
{
  if (done && *done) return;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)K * R) return;
  const int k = (int)(t / R), c = (int)(t - (int64_t)k * R);
  dst[t] = src[(size_t)idx[k] * R + c];
}

// the coordinates each direction's digit kernel reads: (rows, normals,
// sources) with the reduction axis in Morton order
static void oz_coords(const Solver &S, int DIR, const float4 **xr, const float4 **nr, const float4 **ys)
{
  if (DIR == 0) {
    *xr = S.x4();
    *nr = S.n4();
    *ys = (const float4 *)S.m_oz_ys.ptr;
  } else {
    *xr = (const float4 *)S.m_oz_xr.ptr;
    *nr = (const float4 *)S.m_oz_nr.ptr;
    *ys = S.y4();
  }
}

template <int NPH>
static void oz_mma_launch(const oz::OzArgs &a, unsigned grid, cudaStream_t st)
{
  oz::oz_mma_kernel<NPH><<<grid, oz::kThreads, oz::smem_bytes(2 * NPH), st>>>(a);
}

template <int NPH>
static mbc_status oz_allow()
{
  return allow_max_smem(oz::oz_mma_kernel<NPH>, oz::smem_bytes(2 * NPH));
}

// pack the vector block, then the MMA kernel; returns the row tiles (the
// rows of the curvature partials), 0 if the buffers were not prepared
template <int DIR>
static int oz_launch(const Solver &S, int R, const double *vin, double *out, const double *pdot,
                     double *part, const int32_t *done, cudaStream_t st)
{
  const int M = DIR == 0 ? S.nf : S.n;
  const int K = DIR == 0 ? S.n : S.nf;
  const int np = oz::np_for(R), groups = oz::groups_for(R);
  if (S.m_oz_b.bytes < oz::bimg_bytes(K, R) || S.m_oz_bexp.bytes < sizeof(int32_t) * oz::bexp_count(K, R) ||
      S.m_oz_v.bytes < sizeof(double) * (size_t)K * R) {
    S.oz_unprepared = true;
    return 0;
  }
  double *vg = (double *)S.m_oz_v.ptr;
  oz_gather_kernel<<<(unsigned)cdiv((int64_t)K * R, 256), 256, 0, st>>>(K, R, (const int32_t *)S.m_oz_q[DIR].ptr,
                                                                       vin, vg, done);
  oz::oz_pack_b_kernel<<<dim3(oz::nchunks_for(K), groups), 512, 0, st>>>(
      vg, K, R, np, (int8_t *)S.m_oz_b.ptr, S.m_oz_b.bytes, (int32_t *)S.m_oz_bexp.ptr,
      S.m_oz_bexp.bytes / sizeof(int32_t), done, (int32_t *)S.m_err.ptr);
  oz::OzArgs a{};
  const DevMem &planes = S.oz_slab ? S.m_oz_a[0] : S.m_oz_a[DIR];
  a.adig = (const int8_t *)planes.ptr;
  a.aexp = (const int32_t *)S.m_oz_aexp[DIR].ptr;
  a.bimg = (const int8_t *)S.m_oz_b.ptr;
  a.bexp = (const int32_t *)S.m_oz_bexp.ptr;
  a.adig_size = planes.bytes;
  a.bimg_size = S.m_oz_b.bytes;
  a.aexp_size = S.m_oz_aexp[DIR].bytes / sizeof(int32_t);
  a.bexp_size = S.m_oz_bexp.bytes / sizeof(int32_t);
  a.out = out;
  a.M = M;
  a.K = K;
  a.R = R;
  a.groups = groups;
  a.coef = S.op.coef;
  a.pdot = pdot;
  a.part = part;
  a.done = done;
  a.err = (int32_t *)S.m_err.ptr;
  a.wait_limit = S.wait_limit;
  auto mma = [&](int rt0, int tiles) {
    a.rt0 = rt0;
    const unsigned grid = (unsigned)tiles * (unsigned)groups;
    switch (np) {
      case 16: oz_mma_launch<8>(a, grid, st); break;
      case 32: oz_mma_launch<16>(a, grid, st); break;
      case 48: oz_mma_launch<24>(a, grid, st); break;
      case 64: oz_mma_launch<32>(a, grid, st); break;
      case 80: oz_mma_launch<40>(a, grid, st); break;
      default: oz_mma_launch<48>(a, grid, st); break;
    }
  };
  const int tiles = oz::row_tiles(M);
  if (!S.oz_slab) {
    mma(0, tiles);
    S.launches += 3;
  } else {
    // the planes of each slab of rows, then its products
    const int per = S.oz_slab_tiles[DIR];
    const size_t smem = (DIR == 0 ? 1 : 2) * sizeof(float4) * oz::kChunk;
    const float4 *cx, *cn, *cy;
    oz_coords(S, DIR, &cx, &cn, &cy);
    ++S.launches;  // the gather
    for (int r0 = 0; r0 < tiles; r0 += per) {
      const int cnt = std::min(per, tiles - r0);
      oz::oz_digits_kernel<DIR><<<dim3(oz::nchunks_for(K), cnt), 256, smem, st>>>(
          cx, cn, cy, S.nf, S.n, (int8_t *)planes.ptr, planes.bytes,
          (int32_t *)S.m_oz_aexp[DIR].ptr, S.m_oz_aexp[DIR].bytes / sizeof(int32_t), r0, oz::kModeDigits, done,
          (int32_t *)S.m_err.ptr);
      mma(r0, cnt);
      S.launches += 2;
    }
    ++S.launches;
  }
  return tiles;
}

int oz_launch_rows(const Solver &S, int R, const double *v, double *w, const int32_t *done, cudaStream_t st)
{
  return oz_launch<0>(S, R, v, w, nullptr, nullptr, done, st);
}

int oz_launch_cols(const Solver &S, int R, const double *w, double *t, const double *pdot, double *part,
                   const int32_t *done, cudaStream_t st)
{
  return oz_launch<1>(S, R, w, t, pdot, part, done, st);
}

}  // namespace mbc

mbc_status mbc::Solver::ensure_oz(cudaStream_t st, int R)
{
  namespace oz = mbc::oz;
  if (fp64_matvec != MBC_FP64_MATVEC_INT8) return MBC_OK;
  if (op.kind != MBC_OP_POINT_KERNEL) return fail(MBC_UNSUPPORTED, "the INT8 FP64 matvec needs a point-kernel operator");
  if (!oz_ready) {
    const size_t a0 = oz::adig_bytes(nf, n), a1 = oz::adig_bytes(n, nf);
    size_t free_b = 0, total_b = 0;
    MBC_CK(cudaMemGetInfo(&free_b, &total_b));
    MBC_TRY(m_oz_aexp[0].reserve(sizeof(int32_t) * oz::aexp_count(nf, n)));
    MBC_TRY(m_oz_aexp[1].reserve(sizeof(int32_t) * oz::aexp_count(n, nf)));
    const size_t sm0 = sizeof(float4) * oz::kChunk, sm1 = 2 * sizeof(float4) * oz::kChunk;
    MBC_TRY(allow_max_smem(oz::oz_digits_kernel<0>, sm0));
    MBC_TRY(allow_max_smem(oz::oz_digits_kernel<1>, sm1));
    MBC_TRY(oz_allow<8>());
    MBC_TRY(oz_allow<16>());
    MBC_TRY(oz_allow<24>());
    MBC_TRY(oz_allow<32>());
    MBC_TRY(oz_allow<40>());
    MBC_TRY(oz_allow<48>());
    int mode = oz::kModeExps | oz::kModeDigits;
    oz_slab = a0 + a1 + ((size_t)1 << 30) > free_b;
    if (!oz_slab) {
      // concurrent solvers can take the memory between the check and the
      // allocation: fall back to slab mode rather than fail
      if (m_oz_a[0].reserve(a0) != MBC_OK || m_oz_a[1].reserve(a1) != MBC_OK) {
        m_oz_a[0].release();
        m_oz_a[1].release();
        MBC_CK(cudaMemGetInfo(&free_b, &total_b));
        oz_slab = true;
      }
    }
    if (oz_slab) {
      // the planes do not all fit: keep the exponents, and one buffer that
      // holds the planes of a slab of rows, rebuilt for every matvec; leave
      // room for the PCG workspaces (4 GiB or a tenth of the device)
      const size_t keep = std::max((size_t)4 << 30, total_b / 10);
      const size_t budget = std::min<size_t>(free_b > keep ? free_b - keep : 0, (size_t)40 << 30);
      const size_t t0 = (size_t)oz::nks_for(n) * oz::kDigits * oz::kPlaneBytes;   // per rows tile
      const size_t t1 = (size_t)oz::nks_for(nf) * oz::kDigits * oz::kPlaneBytes;  // per columns tile
      if (budget < std::max(t0, t1))
        return fail(MBC_NO_MEMORY, "INT8 matvec: not even one row tile of digit planes fits (" +
                                       std::to_string(std::max(t0, t1) >> 20) + " MiB)");
      oz_slab_tiles[0] = (int)std::min<size_t>(oz::row_tiles(nf), budget / t0);
      oz_slab_tiles[1] = (int)std::min<size_t>(oz::row_tiles(n), budget / t1);
      m_oz_a[1].release();
      MBC_TRY(m_oz_a[0].reserve(std::max(oz_slab_tiles[0] * t0, oz_slab_tiles[1] * t1)));
      mode = oz::kModeExps;  // exponents of every row now; planes per matvec
    }
    // Morton order of the sources (K direction: its reduction axis) and of
    // the collocation rows (K^T direction), and the coordinates in that order
    {
      std::vector<float4> hx(nf), hn(nf), hy(n);
      MBC_CK(cudaMemcpyAsync(hx.data(), x4(), sizeof(float4) * nf, cudaMemcpyDeviceToHost, st));
      MBC_CK(cudaMemcpyAsync(hn.data(), n4(), sizeof(float4) * nf, cudaMemcpyDeviceToHost, st));
      MBC_CK(cudaMemcpyAsync(hy.data(), y4(), sizeof(float4) * n, cudaMemcpyDeviceToHost, st));
      MBC_CK(cudaStreamSynchronize(st));
      std::vector<int32_t> qs(n), qr(nf);
      MBC_TRY(spatial_order(n, (const float *)hy.data(), 4, qs.data()));
      MBC_TRY(spatial_order(nf, (const float *)hx.data(), 4, qr.data()));
      std::vector<float4> sy(n), sx(nf), sn(nf);
      for (int k = 0; k < n; ++k) sy[k] = hy[qs[k]];
      for (int k = 0; k < nf; ++k) {
        sx[k] = hx[qr[k]];
        sn[k] = hn[qr[k]];
      }
      MBC_TRY(m_oz_q[0].reserve(sizeof(int32_t) * n));
      MBC_TRY(m_oz_q[1].reserve(sizeof(int32_t) * nf));
      MBC_TRY(m_oz_ys.reserve(sizeof(float4) * n));
      MBC_TRY(m_oz_xr.reserve(sizeof(float4) * nf));
      MBC_TRY(m_oz_nr.reserve(sizeof(float4) * nf));
      MBC_CK(cudaMemcpyAsync(m_oz_q[0].ptr, qs.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
      MBC_CK(cudaMemcpyAsync(m_oz_q[1].ptr, qr.data(), sizeof(int32_t) * nf, cudaMemcpyHostToDevice, st));
      MBC_CK(cudaMemcpyAsync(m_oz_ys.ptr, sy.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, st));
      MBC_CK(cudaMemcpyAsync(m_oz_xr.ptr, sx.data(), sizeof(float4) * nf, cudaMemcpyHostToDevice, st));
      MBC_CK(cudaMemcpyAsync(m_oz_nr.ptr, sn.data(), sizeof(float4) * nf, cudaMemcpyHostToDevice, st));
      MBC_CK(cudaStreamSynchronize(st));  // the host vectors go out of scope
    }
    DevMem &p0 = m_oz_a[0], &p1 = oz_slab ? m_oz_a[0] : m_oz_a[1];
    const float4 *cx, *cn, *cy;
    oz_coords(*this, 0, &cx, &cn, &cy);
    oz::oz_digits_kernel<0><<<dim3(oz::nchunks_for(n), oz::row_tiles(nf)), 256, sm0, st>>>(
        cx, cn, cy, nf, n, (int8_t *)p0.ptr, p0.bytes, (int32_t *)m_oz_aexp[0].ptr,
        m_oz_aexp[0].bytes / sizeof(int32_t), 0, mode, nullptr, (int32_t *)m_err.ptr);
    oz_coords(*this, 1, &cx, &cn, &cy);
    oz::oz_digits_kernel<1><<<dim3(oz::nchunks_for(nf), oz::row_tiles(n)), 256, sm1, st>>>(
        cx, cn, cy, nf, n, (int8_t *)p1.ptr, p1.bytes, (int32_t *)m_oz_aexp[1].ptr,
        m_oz_aexp[1].bytes / sizeof(int32_t), 0, mode, nullptr, (int32_t *)m_err.ptr);
    launches += 2;
    MBC_CKL();
    MBC_TRY(check_device_error(st));
    const int K = std::max(n, nf);
    MBC_TRY(m_oz_b.reserve(oz::bimg_bytes(K, std::max(R, 1))));
    MBC_TRY(m_oz_bexp.reserve(sizeof(int32_t) * oz::bexp_count(K, std::max(R, 1))));
    MBC_TRY(m_oz_v.reserve(sizeof(double) * (size_t)K * std::max(R, 1)));
    MBC_TRY(oz_selfcheck(st));
  }
  const int K = std::max(n, nf);
  MBC_TRY(m_oz_b.reserve(oz::bimg_bytes(K, R)));
  MBC_TRY(m_oz_bexp.reserve(sizeof(int32_t) * oz::bexp_count(K, R)));
  MBC_TRY(m_oz_v.reserve(sizeof(double) * (size_t)K * R));
  return MBC_OK;
}

mbc_status mbc::Solver::oz_selfcheck(cudaStream_t st)
{
  // a wrong plane or kernel shows as an O(1) difference; the scheme's own
  // error is ~1e-10 relative, so 1e-8 leaves a wide margin
  const double tol = 1e-8;
  MBC_TRY(m_oz_chk.reserve(sizeof(double) * (3 * (size_t)n + 2 * (size_t)nf)));
  double *v = (double *)m_oz_chk.ptr, *t8 = v + n, *t64 = t8 + n, *w8 = t64 + n, *w64 = w8 + nf;
  std::vector<double> hv(n);
  uint64_t x = 0x9E3779B97F4A7C15ull;  // a fixed LCG sequence in [-1, 1)
  for (double &e : hv) {
    x = x * 6364136223846793005ull + 1442695040888963407ull;
    e = (double)(x >> 11) * 0x1p-53 * 2.0 - 1.0;
  }
  MBC_CK(cudaMemcpyAsync(v, hv.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st));
  oz_ready = true;
  launch_rows<double>(*this, 1, v, w8, nullptr, st);
  launch_cols<double>(*this, 1, w8, t8, nullptr, nullptr, nullptr, st);
  fp64_matvec = MBC_FP64_MATVEC_SIMT;
  launch_rows<double>(*this, 1, v, w64, nullptr, st);
  launch_cols<double>(*this, 1, w8, t64, nullptr, nullptr, nullptr, st);
  fp64_matvec = MBC_FP64_MATVEC_INT8;
  MBC_CKL();
  mbc_status e = check_device_error(st);
  if (e != MBC_OK) {
    oz_ready = false;
    return e;
  }
  std::vector<double> h((size_t)2 * n + 2 * (size_t)nf);
  MBC_CK(cudaMemcpyAsync(h.data(), t8, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st));
  MBC_CK(cudaStreamSynchronize(st));
  auto rel = [](const double *a, const double *b, size_t m) {
    double d = 0, r = 0;
    for (size_t i = 0; i < m; ++i) {
      d += (a[i] - b[i]) * (a[i] - b[i]);
      r += b[i] * b[i];
    }
    return r > 0 ? std::sqrt(d / r) : std::sqrt(d);
  };
  const double dk = rel(h.data() + 2 * (size_t)n, h.data() + 2 * (size_t)n + nf, nf);  // w8 vs w64
  const double dkt = rel(h.data(), h.data() + n, n);                                     // t8 vs t64
  if (!(dk <= tol) || !(dkt <= tol)) {
    oz_ready = false;
    return fail(MBC_CUDA_ERROR, "INT8 matvec self-check failed: relative difference to the FP64 kernels " +
                                    std::to_string(dk) + " (K), " + std::to_string(dkt) + " (K^T)");
  }
  return MBC_OK;
}

using mbc::fail;

extern "C" mbc_status mbc_solver_set_fp64_matvec(mbc_solver *s, int32_t impl)
{
  if (!s) return fail(MBC_BAD_ARG, "NULL solver");
  if (impl != MBC_FP64_MATVEC_SIMT && impl != MBC_FP64_MATVEC_INT8) return fail(MBC_BAD_ARG, "unknown FP64 matvec implementation");
  if (impl == MBC_FP64_MATVEC_INT8 && s->s.op.kind != MBC_OP_POINT_KERNEL)
    return fail(MBC_UNSUPPORTED, "the INT8 FP64 matvec needs a point-kernel operator");
  s->s.fp64_matvec = impl;
  return MBC_OK;
}

extern "C" mbc_status mbc_solver_prepare(mbc_solver *s, mbc_stream stream)
{
  if (!s) return fail(MBC_BAD_ARG, "NULL solver");
  MBC_TRY(s->s.ensure_oz((cudaStream_t)stream, 1));
  MBC_CK(cudaStreamSynchronize((cudaStream_t)stream));
  return MBC_OK;
}

