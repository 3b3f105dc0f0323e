// Device solver for the MFS solve path: operator storage, supernodal KL
// factor and batched PCG, behind the C ABI in include/mbc.h.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <type_traits>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "block.cuh"
#include "factor.cuh"
#include "factor_tc.cuh"
#include "forces.cuh"
#include "matvec.cuh"
#include "matvec_mesh.cuh"
#include "matvec_tc.cuh"
#include "cuda_util.h"
#include "int8_ops.h"
#include "mbc_internal.h"
#include "pcg.cuh"
#include "solver.h"

namespace mbc {

DevMem::~DevMem() { release(); }
void DevMem::release()
{
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
}
mbc_status DevMem::reserve(size_t b)
{
  if (b <= bytes && ptr) return MBC_OK;
  release();
  if (b == 0) b = 16;
  cudaError_t e = cudaMalloc(&ptr, b);
  if (e != cudaSuccess) {
    ptr = nullptr;
    cudaGetLastError();
    return fail(MBC_NO_MEMORY, std::string("cudaMalloc(") + std::to_string(b) + "): " + cudaGetErrorString(e));
  }
  bytes = b;
  return MBC_OK;
}

template <typename V>
static mbc_status upload(DevMem &m, const std::vector<V> &h, cudaStream_t st)
{
  MBC_TRY(m.reserve(std::max<size_t>(h.size() * sizeof(V), 16)));
  if (!h.empty()) MBC_CK(cudaMemcpyAsync(m.ptr, h.data(), h.size() * sizeof(V), cudaMemcpyHostToDevice, st));
  return MBC_OK;
}

// --------------------------------------------------------------------------
// matvec dispatch
// --------------------------------------------------------------------------
namespace {

constexpr int TJ_ROWS = 128;
constexpr int TJ_COLS = 64;

// Launch shape for a direction with `rows` outputs and R columns: the widest
// column chunk RC (fewest kernel re-evaluations) and the larger block TI that
// still give at least four blocks per SM; otherwise the shape with the most
// blocks.
struct Shape {
  int ti, rc;
};

template <typename T>
Shape pick_shape(int rows, int R)
{
  const int want = 4 * 148;
  if (R == 1) return {rows >= 128 * want ? 128 : 64, 1};
  static const Shape f32[] = {{128, 64}, {128, 32}, {64, 32}, {64, 16}, {64, 8}, {64, 4}};
  static const Shape f64[] = {{128, 32}, {64, 32}, {64, 16}, {64, 8}, {64, 4}};
  const Shape *c = sizeof(T) == 8 ? f64 : f32;
  const int nc = sizeof(T) == 8 ? 5 : 6;
  Shape best = c[0];
  int64_t best_blocks = -1;
  for (int k = 0; k < nc; ++k) {
    if (c[k].rc > 4 && c[k].rc / 2 >= R) continue;  // chunk much wider than R
    const int64_t blocks = (int64_t)cdiv(rows, c[k].ti) * cdiv(R, c[k].rc);
    if (blocks >= want) return c[k];
    if (blocks > best_blocks) {
      best = c[k];
      best_blocks = blocks;
    }
  }
  return best;
}

template <typename T, int RC, int TI>
void rows_launch(const Solver &S, int R, const T *v, T *w, const int32_t *done, cudaStream_t st)
{
  if (S.op.kind == MBC_OP_POINT_KERNEL) {
    dim3 grid(cdiv(S.nf, TI), cdiv(R, RC));
    pk_rows_kernel<T, RC, TI, TJ_ROWS><<<grid, TI, 0, st>>>(S.x4(), S.n4(), S.nf, S.y4(), S.n, v, R,
                                                            (T)S.op.coef, w, R, R, done);
  } else if (S.op.kind == MBC_OP_MESH) {
    dim3 grid(cdiv(S.nf, TI), cdiv(R, RC));
    mesh_rows_kernel<T, RC, TI, TJ_ROWS><<<grid, TI, 0, st>>>(S.x4(), S.n4(), S.z4(), S.nf, S.y4(), S.n, v, R,
                                                              (T)S.op.coef, w, R, R, done);
  } else {
    dim3 grid(cdiv(S.nf, 8), cdiv(R, RC));
    dense_rows_kernel<T, RC><<<grid, 256, 0, st>>>(S.op.M, S.op.ldm, S.nf, S.n, S.dP(), v, R, w,
                                                    R, R, done);
  }
}

template <typename T, int RC, int TI>
int cols_launch(const Solver &S, int R, const T *w, T *t, const T *pdot, double *part,
                const int32_t *done, cudaStream_t st)
{
  dim3 grid(cdiv(S.n, TI), cdiv(R, RC));
  if (S.op.kind == MBC_OP_POINT_KERNEL) {
    pk_cols_kernel<T, RC, TI, TJ_COLS><<<grid, TI, 0, st>>>(S.x4(), S.n4(), S.nf, S.y4(), S.n, w, R,
                                                            (T)S.op.coef, t, R, R, pdot, part, done);
  } else if (S.op.kind == MBC_OP_MESH) {
    mesh_cols_kernel<T, RC, TI, TJ_COLS><<<grid, TI, 0, st>>>(S.x4(), S.n4(), S.z4(), S.nf, S.y4(), S.n, w, R,
                                                              (T)S.op.coef, t, R, R, pdot, part, done);
  } else {
    dense_cols_kernel<T, RC, TI, 32><<<grid, TI, 0, st>>>(S.op.M, S.op.ldm, S.nf, S.n, S.dP(), w, R,
                                                          t, R, R, pdot, part, done);
  }
  return (int)grid.x;
}

}  // namespace

// tensor-core path: FP32 point kernel, R <= 256 (auto: R >= 8); needs the
// packed B image buffer (falls back to the CUDA-core kernels without it)
static bool use_tc(const Solver &S, int R)
{
  if (S.op.kind != MBC_OP_POINT_KERNEL || R > 256) return false;
  if (S.matvec_impl == MBC_MATVEC_SIMT) return false;
  if (S.matvec_impl == MBC_MATVEC_AUTO && R < 8) return false;
  const int np = (R + 15) / 16 * 16;
  const int K = std::max(S.n, S.nf);
  const size_t need = (size_t)cdiv(K, tc::kK) * 2 * tc::tile_b_bytes(np);
  // both directions must fit the device's shared memory (true on sm_100a)
  if (allow_max_smem(tc::pk_tc_kernel<0>, tc::smem_bytes(np, 0)) != MBC_OK ||
      allow_max_smem(tc::pk_tc_kernel<1>, tc::smem_bytes(np, 1)) != MBC_OK)
    return false;
  return S.m_bimg.reserve(need) == MBC_OK;
}

template <int DIR>
static int tc_launch(const Solver &S, int R, const float *vin, float *out, const float *pdot,
                     double *part, const int32_t *done, cudaStream_t st)
{
  const int M = DIR == 0 ? S.nf : S.n;
  const int K = DIR == 0 ? S.n : S.nf;
  tc::TcArgs a{};
  a.xr = S.x4();
  a.nr = S.n4();
  a.ys = S.y4();
  a.nf = S.nf;
  a.n = S.n;
  a.bimg = (const uint4 *)S.m_bimg.ptr;
  a.out = out;
  a.R = R;
  a.np = (R + 15) / 16 * 16;
  a.tmem_cols = tc::tmem_cols_for(a.np);
  a.coef = (float)S.op.coef;
  a.pdot = pdot;
  a.part = part;
  a.done = done;
  a.err = (int32_t *)S.m_err.ptr;
  a.wait_limit = S.wait_limit;
  const int nks = (int)cdiv(K, tc::kK);
  const int64_t pack_threads = (int64_t)nks * a.np * (tc::kK / 4);
  tc::pack_b_kernel<<<cdiv(pack_threads, 256), 256, 0, st>>>(vin, K, R, a.np, nks, (uint4 *)S.m_bimg.ptr,
                                                              done);
  const int smem = tc::smem_bytes(a.np, DIR);  // allowed by use_tc
  const unsigned grid = cdiv(M, tc::kM);
  tc::pk_tc_kernel<DIR><<<grid, tc::kThreads, smem, st>>>(a);
  return (int)grid;
}

#define MBC_SHAPES(T, X)                                                   \
  X(T, 1, 64) X(T, 1, 128) X(T, 4, 64) X(T, 8, 64) X(T, 16, 64) X(T, 32, 64) X(T, 32, 128)

template <typename T>
void launch_rows(const Solver &S, int R, const T *v, T *w, const int32_t *done, cudaStream_t st)
{
  if constexpr (sizeof(T) == 4) {
    if (use_tc(S, R)) {
      tc_launch<0>(S, R, v, w, nullptr, nullptr, done, st);
      S.launches += 2;
      return;
    }
  } else {
    if (use_oz(S)) {
      oz_launch_rows(S, R, v, w, done, st);
      return;
    }
  }
  ++S.launches;
  const Shape sh = pick_shape<T>(S.op.kind != MBC_OP_DENSE ? S.nf : 1 << 30, R);
#define MBC_ROWS_CASE(TT, RC_, TI_) \
  if (sh.rc == RC_ && sh.ti == TI_) return rows_launch<T, RC_, TI_>(S, R, v, w, done, st);
  MBC_SHAPES(T, MBC_ROWS_CASE)
  if constexpr (sizeof(T) == 4) {
    if (sh.rc == 64) return rows_launch<T, 64, 128>(S, R, v, w, done, st);
  }
#undef MBC_ROWS_CASE
  rows_launch<T, 32, 64>(S, R, v, w, done, st);
}

template <typename T>
int launch_cols(const Solver &S, int R, const T *w, T *t, const T *pdot, double *part,
                const int32_t *done, cudaStream_t st)
{
  if constexpr (sizeof(T) == 4) {
    if (use_tc(S, R)) {
      S.launches += 2;
      return tc_launch<1>(S, R, w, t, pdot, part, done, st);
    }
  } else {
    if (use_oz(S)) return oz_launch_cols(S, R, w, t, pdot, part, done, st);
  }
  ++S.launches;
  const Shape sh = pick_shape<T>(S.n, R);
#define MBC_COLS_CASE(TT, RC_, TI_) \
  if (sh.rc == RC_ && sh.ti == TI_) return cols_launch<T, RC_, TI_>(S, R, w, t, pdot, part, done, st);
  MBC_SHAPES(T, MBC_COLS_CASE)
  if constexpr (sizeof(T) == 4) {
    if (sh.rc == 64) return cols_launch<T, 64, 128>(S, R, w, t, pdot, part, done, st);
  }
#undef MBC_COLS_CASE
  return cols_launch<T, 32, 64>(S, R, w, t, pdot, part, done, st);
}

// upper bound on the blocks of any columns-direction launch (the per-block
// curvature partials): SIMT tiles of 64 sources or more, tensor cores 128
int cols_blocks(const Solver &S) { return (int)cdiv(S.n, 64); }

template void launch_rows<float>(const Solver &, int, const float *, float *, const int32_t *, cudaStream_t);
template void launch_rows<double>(const Solver &, int, const double *, double *, const int32_t *, cudaStream_t);
template int launch_cols<float>(const Solver &, int, const float *, float *, const float *, double *, const int32_t *, cudaStream_t);
template int launch_cols<double>(const Solver &, int, const double *, double *, const double *, double *, const int32_t *, cudaStream_t);

// --------------------------------------------------------------------------
// factor
// --------------------------------------------------------------------------
namespace {

// FP32 supernodes whose pivots cancel below this fraction of their diagonal
// (more than ~3 of FP32's ~7 digits lost) are refactored in FP64.
constexpr double kF32PivotTol = 1e-3;
// threads per class; the class bounds and panel rows come from the solver's
// mbc_factor_tiles (default: n_s <= 32, <= 64, <= 128 in shared memory,
// larger ones in global memory; 64, 32, 32, 8 panel rows)
constexpr int kClassThreads[4] = {128, 256, 512, 512};

// the dynamic shared memory a block may opt in to on this device
static int smem_optin_cap()
{
  int dev = 0, cap = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 48 * 1024;
  if (cudaDeviceGetAttribute(&cap, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 48 * 1024;
  return cap - 1024;  // room for the kernel's static shared variables
}

template <typename T>
size_t factor_smem(int ns_max, int nt, int tr, bool theta_in_smem)
{
  auto al = [](size_t b) { return (b + 15) & ~(size_t)15; };
  size_t b = al((size_t)ns_max * sizeof(float4)) + al((size_t)tr * ns_max * sizeof(T));
  if (theta_in_smem) b += al((size_t)(nt / 32) * ns_max * sizeof(T)) + (size_t)ns_max * ns_max * sizeof(T);
  return b;
}

template <typename T, typename LT, int NT, int EPT>
mbc_status launch_factor_class(FactorArgs a, T *theta, LT *lval, size_t smem, cudaStream_t st)
{
  auto kern = factor_kernel<T, LT, NT, EPT>;
  MBC_TRY(allow_max_smem(kern, smem));
  kern<<<a.count, NT, smem, st>>>(a, theta, lval);
  MBC_CKL();
  return MBC_OK;
}

}  // namespace

// Theta of the listed supernodes (FP32) by the tensor-core Gram kernel
static mbc_status launch_gram(Solver &S, const std::vector<int32_t> &gram, float *theta, cudaStream_t st)
{
  MBC_TRY(upload(S.gram_list, gram, st));
  ftc::GramArgs g{};
  g.list = (const int32_t *)S.gram_list.ptr;
  g.count = (int32_t)gram.size();
  g.set_ptr = S.d_set_ptr();
  g.set_ind = S.d_set_ind();
  g.th_ptr = S.d_th_ptr();
  g.kind = S.op.kind;
  g.xr = S.x4();
  g.nr = S.n4();
  g.zr = S.z4();
  g.ys = S.y4();
  g.M = S.op.M;
  g.ldm = S.op.ldm;
  g.Pinv = S.d_Pinv();
  g.nf = S.nf;
  g.coef = (float)S.op.coef;
  g.theta = theta;
  g.err = (int32_t *)S.m_err.ptr;
  g.wait_limit = S.wait_limit;
  MBC_TRY(allow_max_smem(ftc::gram_tc_kernel, ftc::smem_bytes()));
  ftc::gram_tc_kernel<<<(unsigned)gram.size(), ftc::kThreads, ftc::smem_bytes(), st>>>(g);
  ++S.launches;
  MBC_CKL();
  S.gram_tc_count += (int32_t)gram.size();
  return MBC_OK;
}

// Launch the factor kernels over the given per-class supernode lists.  In
// FP32 the supernodes with tiles.tc_min_ns <= n_s <= ftc::kMaxNs take their
// Gram from the tensor cores first (tc_min_ns = 0: none).
template <typename T, typename LT>
static mbc_status run_factor(Solver &S, const std::vector<int32_t> *lists, T *theta, LT *lval,
                             double shift, double pivot_tol, int32_t *d_bad_list,
                             int32_t *d_bad_count, cudaStream_t st)
{
  const Plan &p = *S.plan;
  std::vector<int32_t> simt[4], tcl[4], gram;
  const int tc_min = std::is_same<T, float>::value ? S.tiles.tc_min_ns : 0;
  for (int c = 0; c < 4; ++c)
    for (int32_t s : lists[c]) {
      const int ns = p.set_ptr[s + 1] - p.set_ptr[s];
      if (tc_min > 0 && ns >= tc_min && ns <= ftc::kMaxNs) {
        tcl[c].push_back(s);
        gram.push_back(s);
      } else {
        simt[c].push_back(s);
      }
    }
  if constexpr (std::is_same<T, float>::value)
    if (!gram.empty()) MBC_TRY(launch_gram(S, gram, theta, st));
  for (int job = 0; job < 8; ++job) {
    const int c = job & 3, ready = job >> 2;
    const auto &lst = ready ? tcl[c] : simt[c];
    if (lst.empty()) continue;
    DevMem &dl = ready ? S.class_list_tc[c] : S.class_list[c];
    MBC_TRY(upload(dl, lst, st));
    int ns_max = 0;
    for (int32_t s : lst) ns_max = std::max(ns_max, p.set_ptr[s + 1] - p.set_ptr[s]);
    FactorArgs a{};
    a.list = (const int32_t *)dl.ptr;
    a.count = (int32_t)lst.size();
    a.sup_ptr = S.d_sup_ptr();
    a.sup_ind = S.d_sup_ind();
    a.set_ptr = S.d_set_ptr();
    a.set_ind = S.d_set_ind();
    a.lptr = S.d_lptr();
    a.th_ptr = S.d_th_ptr();
    a.kind = S.op.kind;
    a.xr = S.x4();
    a.nr = S.n4();
    a.zr = S.z4();
    a.ys = S.y4();
    a.M = S.op.M;
    a.ldm = S.op.ldm;
    a.Pinv = S.d_Pinv();
    a.nf = S.nf;
    a.coef = S.op.coef;
    a.shift = shift;
    a.pivot_tol = pivot_tol;
    a.gram_ready = ready;
    a.bad_list = d_bad_list;
    a.bad_count = d_bad_count;
    const int nt = kClassThreads[c];
    const bool in_smem = c < 3;
    int tr = std::max(1, S.tiles.tile_rows[c]);
    if (!in_smem) {
      tr = (int)std::max<int64_t>(1, std::min<int64_t>(tr, (96 * 1024) / ((int64_t)ns_max * sizeof(T))));
      MBC_TRY(S.fscratch.reserve((size_t)lst.size() * (nt / 32) * ns_max * sizeof(T)));
      a.gscratch = S.fscratch.ptr;
      a.gscratch_stride = ns_max;
    }
    // fewer panel rows where the class's Theta and buffers leave too little
    // shared memory (the FP64 retries need twice the FP32 launch's)
    const size_t cap = (size_t)smem_optin_cap();
    while (tr > 1 && factor_smem<T>(ns_max, nt, tr, in_smem) > cap) tr /= 2;
    a.smem_cap = in_smem ? S.tiles.max_ns[c] : 0;
    a.tile_rows = tr;
    const size_t smem = factor_smem<T>(ns_max, nt, tr, in_smem);
    switch (c) {
      case 0: MBC_TRY((launch_factor_class<T, LT, 128, 5>(a, theta, lval, smem, st))); break;
      case 1: MBC_TRY((launch_factor_class<T, LT, 256, 9>(a, theta, lval, smem, st))); break;
      case 2: MBC_TRY((launch_factor_class<T, LT, 512, 17>(a, theta, lval, smem, st))); break;
      default: MBC_TRY((launch_factor_class<T, LT, 512, 16>(a, theta, lval, smem, st))); break;
    }
  }
  return MBC_OK;
}

static void split_classes(const Plan &p, const mbc_factor_tiles &t, const std::vector<int32_t> &ids,
                          std::vector<int32_t> *lists)
{
  for (int c = 0; c < 4; ++c) lists[c].clear();
  for (int32_t s : ids) {
    const int ns = p.set_ptr[s + 1] - p.set_ptr[s];
    int c = 3;
    for (int k = 0; k < 3; ++k)
      if (ns <= t.max_ns[k]) {
        c = k;
        break;
      }
    lists[c].push_back(s);
  }
  // largest first inside a class: the long CTAs start early
  for (int c = 0; c < 4; ++c)
    std::stable_sort(lists[c].begin(), lists[c].end(), [&](int32_t a, int32_t b) {
      return p.set_ptr[a + 1] - p.set_ptr[a] > p.set_ptr[b + 1] - p.set_ptr[b];
    });
}

mbc_status Solver::factor(cudaStream_t st)
{
  const Plan &p = *plan;
  const size_t th_n = (size_t)p.th_ptr.back();
  const size_t l_n = (size_t)p.lptr.back();
  const size_t esz = precision == MBC_F64 ? 8 : 4;
  MBC_TRY(theta.reserve(std::max<size_t>(th_n * esz, 16)));
  MBC_TRY(lval.reserve(std::max<size_t>(l_n * esz, 16)));
  MBC_TRY(bad.reserve(sizeof(int32_t) * (p.n_super + 1)));
  MBC_CK(cudaMemsetAsync(bad.ptr, 0, sizeof(int32_t), st));
  int32_t *d_bad_count = (int32_t *)bad.ptr;
  int32_t *d_bad_list = d_bad_count + 1;
  std::vector<int32_t> all(p.n_super);
  for (int32_t s = 0; s < p.n_super; ++s) all[s] = s;
  std::vector<int32_t> lists[4];
  split_classes(p, tiles, all, lists);
  gram_tc_count = 0;
  if (precision == MBC_F64)
    MBC_TRY((run_factor<double, double>(*this, lists, (double *)theta.ptr, (double *)lval.ptr, 0.0,
                                        0.0, d_bad_list, d_bad_count, st)));
  else
    MBC_TRY((run_factor<float, float>(*this, lists, (float *)theta.ptr, (float *)lval.ptr, 0.0,
                                      kF32PivotTol, d_bad_list, d_bad_count, st)));
  // a tensor-core Gram that stopped on a bounded wait left its Theta unwritten
  if (gram_tc_count > 0) MBC_TRY(check_device_error(st));
  // supernodes with a non-positive pivot: redo in FP64, then FP64 with a
  // small diagonal shift
  pivot_retries = 0;
  const double shifts[2] = {0.0, 1e-10};
  for (int attempt = 0; attempt < 2; ++attempt) {
    int32_t nbad = 0;
    MBC_CK(cudaMemcpyAsync(&nbad, d_bad_count, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    MBC_CK(cudaStreamSynchronize(st));
    if (nbad == 0) break;
    if (precision == MBC_F64 && attempt == 0) continue;  // FP64 already: go to the shift
    std::vector<int32_t> ids(nbad);
    MBC_CK(cudaMemcpy(ids.data(), d_bad_list, sizeof(int32_t) * nbad, cudaMemcpyDeviceToHost));
    pivot_retries += nbad;
    MBC_CK(cudaMemsetAsync(d_bad_count, 0, sizeof(int32_t), st));
    split_classes(p, tiles, ids, lists);
    MBC_TRY(theta64.reserve(std::max<size_t>(th_n * 8, 16)));
    if (precision == MBC_F64)
      MBC_TRY((run_factor<double, double>(*this, lists, (double *)theta.ptr, (double *)lval.ptr,
                                          shifts[attempt], 0.0, d_bad_list, d_bad_count, st)));
    else
      MBC_TRY((run_factor<double, float>(*this, lists, (double *)theta64.ptr, (float *)lval.ptr,
                                         shifts[attempt], 0.0, d_bad_list, d_bad_count, st)));
  }
  {
    int32_t nbad = 0;
    MBC_CK(cudaMemcpyAsync(&nbad, d_bad_count, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    MBC_CK(cudaStreamSynchronize(st));
    if (nbad > 0) {
      // the shifted FP64 retry also failed: count it but keep its columns
      // from the retry (precision F64 shifts directly); report the status
      factored = false;
      return fail(MBC_NONSPD_PIVOT, std::to_string(nbad) + " supernode(s) not positive definite");
    }
  }
  factored = true;
  return MBC_OK;
}

// --------------------------------------------------------------------------
// solver creation
// --------------------------------------------------------------------------
mbc_status Solver::create(const Plan &pl, const mbc_operator &o, int32_t prec, cudaStream_t st)
{
  plan = &pl;
  op = o;
  precision = prec;
  n = pl.n;
  nf = o.nf;
  MBC_TRY(upload(m_P, pl.P, st));
  MBC_TRY(upload(m_Pinv, pl.Pinv, st));
  MBC_TRY(upload(m_sup_ptr, pl.sup_ptr, st));
  MBC_TRY(upload(m_sup_ind, pl.sup_ind, st));
  MBC_TRY(upload(m_set_ptr, pl.set_ptr, st));
  MBC_TRY(upload(m_set_ind, pl.set_ind, st));
  MBC_TRY(upload(m_lptr, pl.lptr, st));
  MBC_TRY(upload(m_lind, pl.lind, st));
  MBC_TRY(upload(m_rptr, pl.rptr, st));
  MBC_TRY(upload(m_rcol, pl.rcol, st));
  MBC_TRY(upload(m_rmap, pl.rmap, st));
  MBC_TRY(upload(m_th_ptr, pl.th_ptr, st));
  MBC_TRY(m_err.reserve(sizeof(int32_t)));
  MBC_CK(cudaMemsetAsync(m_err.ptr, 0, sizeof(int32_t), st));
  if (o.kind == MBC_OP_MESH) {
    // faces as three vertex arrays (original face order), sources in plan order
    MBC_TRY(m_x4.reserve(sizeof(float4) * nf));
    MBC_TRY(m_n4.reserve(sizeof(float4) * nf));
    MBC_TRY(m_z4.reserve(sizeof(float4) * nf));
    MBC_TRY(m_y4.reserve(sizeof(float4) * n));
    pack_faces_kernel<<<cdiv(nf, 256), 256, 0, st>>>(nf, o.V, o.n_vert, o.faces, (float4 *)m_x4.ptr,
                                                     (float4 *)m_n4.ptr, (float4 *)m_z4.ptr);
    pack_points_kernel<<<cdiv(n, 256), 256, 0, st>>>(n, o.y, (const int32_t *)m_Pinv.ptr, (float4 *)m_y4.ptr);
    MBC_CKL();
  }
  if (o.kind == MBC_OP_POINT_KERNEL) {
    // padded to whole 32-point tiles (the tensor-core path copies whole tiles)
    const size_t nf_pad = (size_t)cdiv(nf, 32) * 32, n_pad = (size_t)cdiv(n, 32) * 32;
    MBC_TRY(m_x4.reserve(sizeof(float4) * nf_pad));
    MBC_TRY(m_n4.reserve(sizeof(float4) * nf_pad));
    MBC_TRY(m_y4.reserve(sizeof(float4) * n_pad));
    MBC_CK(cudaMemsetAsync(m_x4.ptr, 0, sizeof(float4) * nf_pad, st));
    MBC_CK(cudaMemsetAsync(m_n4.ptr, 0, sizeof(float4) * nf_pad, st));
    MBC_CK(cudaMemsetAsync(m_y4.ptr, 0, sizeof(float4) * n_pad, st));
    pack_points_kernel<<<cdiv(nf, 256), 256, 0, st>>>(nf, o.x, nullptr, (float4 *)m_x4.ptr);
    pack_points_kernel<<<cdiv(nf, 256), 256, 0, st>>>(nf, o.nx, nullptr, (float4 *)m_n4.ptr);
    pack_points_kernel<<<cdiv(n, 256), 256, 0, st>>>(n, o.y, (const int32_t *)m_Pinv.ptr,
                                                     (float4 *)m_y4.ptr);
    MBC_CKL();
  }
  MBC_CK(cudaStreamSynchronize(st));
  return MBC_OK;
}

// --------------------------------------------------------------------------
// PCG
// --------------------------------------------------------------------------
namespace {

struct Layout2D {
  dim3 block, grid;
  size_t smem;
};

Layout2D layout2d(int n, int R)
{
  int bx = 1;
  while (bx < R && bx < 32) bx <<= 1;
  const int by = 256 / bx;
  Layout2D L;
  L.block = dim3(bx, by);
  L.grid = dim3(cdiv(n, by), cdiv(R, bx));
  L.smem = sizeof(double) * 256;
  return L;
}

}  // namespace

// Work buffers for one precision.  X64 is the FP64 solution accumulator of
// the residual-replacement mode.
template <typename T>
struct PcgWork {
  T *X, *Rv, *Pv, *Z, *U, *Tt, *W;
  double *X64 = nullptr;
  double *part;
  int part_stride;  // blocks
  PcgScalars sc;
};

// PCG buffers for R columns in the given storage (vectors, block partials,
// per-column scalars)
template <typename T>
static mbc_status pcg_buffers_in(Solver &S, int R, PcgWork<T> &w, DevMem &m, DevMem &part, DevMem &scal)
{
  const size_t nv = (size_t)S.n * R, fv = (size_t)S.nf * R;
  const size_t vb = ((nv * sizeof(T)) + 255) & ~(size_t)255;
  const size_t fb = ((fv * sizeof(T)) + 255) & ~(size_t)255;
  MBC_TRY(m.reserve(6 * vb + fb));
  char *b = (char *)m.ptr;
  w.X = (T *)b;
  w.Rv = (T *)(b + vb);
  w.Pv = (T *)(b + 2 * vb);
  w.Z = (T *)(b + 3 * vb);
  w.U = (T *)(b + 4 * vb);
  w.Tt = (T *)(b + 5 * vb);
  w.W = (T *)(b + 6 * vb);
  const int nblk = std::max<int>(std::max<int>(cols_blocks(S), layout2d(S.n, R).grid.x), 1);
  w.part_stride = nblk;
  MBC_TRY(part.reserve(sizeof(double) * (size_t)nblk * R));
  w.part = (double *)part.ptr;
  MBC_TRY(scal.reserve(sizeof(double) * 8 * R + sizeof(int32_t) * (3 * R + 4)));
  double *d = (double *)scal.ptr;
  w.sc.rz = d;
  w.sc.b2 = d + R;
  w.sc.thr = d + 2 * R;
  w.sc.alpha = d + 3 * R;
  w.sc.beta = d + 4 * R;
  w.sc.rr = d + 5 * R;
  w.sc.pt = d + 6 * R;
  w.sc.rr_ref = d + 7 * R;
  int32_t *ii = (int32_t *)(d + 8 * R);
  w.sc.status = ii;
  w.sc.iters = ii + R;
  w.sc.done = ii + 2 * R;
  w.sc.want = ii + 2 * R + 1;
  w.sc.stall = ii + 2 * R + 4;
  w.sc.drop2 = 0.0;
  w.sc.stall_check = 1;
  return MBC_OK;
}

template <typename T>
static mbc_status pcg_buffers(Solver &S, int R, PcgWork<T> &w)
{
  return pcg_buffers_in<T>(S, R, w, sizeof(T) == 8 ? S.work64 : S.work32, S.part, S.scal);
}

__global__ void set_status_kernel(int R, int32_t *status, int32_t *iters, int32_t *done,
                                  int32_t *want, double *rz, const int32_t *mask)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c == 0) {
    *done = 0;
    *want = 0;
  }
  if (c >= R) return;
  status[c] = (mask == nullptr || mask[c]) ? COL_ACTIVE : COL_OK;
  iters[c] = 0;
  rz[c] = __longlong_as_double(0x7ff0000000000000LL);  // +inf: the first beta is 0
}

// Warm starts: thresholds relative to |b|^2 of the original right-hand side.
__global__ void set_thresholds_kernel(int R, double tol2, const double *b2ref, PcgScalars sc)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= R) return;
  sc.b2[c] = b2ref[c];
  sc.thr[c] = tol2 * b2ref[c];
  if (b2ref[c] < 1e-16 && sc.status[c] == COL_ACTIVE) sc.status[c] = COL_OK;
}

// Run PCG on (K^T K) x = b for R columns (the recurrences of kl_chol.cu:975-1078
// per column).  On entry w.Rv holds the residual b - K^T K x of the start x
// (x = w.X, or w.X64 when `replace` is given).  One iteration here is
//   z = L L^T r, beta = r.z / rz_old, p = z + beta p, t = K^T K p,
//   alpha = r.z / p.t, x += alpha p, r -= alpha t, stop test on |r|^2,
// so a host check point falls right after the residual update: that is
// where `replace` (residual replacement) swaps in the FP64 true residual,
// keeping p and therefore the Krylov information.
template <typename T, typename LT, typename XT>
static mbc_status run_pcg(Solver &S, int R, PcgWork<T> &w, XT *x, const LT *lval, int maxit,
                          double tol, bool precond, int check_every, const int32_t *d_mask,
                          cudaStream_t st, const double *d_b2ref,
                          const std::function<mbc_status()> *replace, int max_replace, bool compact = false)
{
  // Blocks of check_every iterations have fixed kernel arguments (scalars
  // live on the device), so with S.graph a full block is captured once as a
  // CUDA graph and replayed: one launch per block instead of ~9 per
  // iteration, which matters for small scenes.  The first block runs
  // eagerly (it sizes every buffer); profiling runs eagerly throughout.
  struct GraphGuard {
    cudaGraphExec_t exec = nullptr;
    ~GraphGuard()
    {
      if (exec) cudaGraphExecDestroy(exec);
    }
  } graph;
  int64_t graph_launches = 0;
  const Layout2D L = layout2d(S.n, R);
  const int nblk2 = (int)L.grid.x;
  w.sc.maxit = maxit;
  w.sc.tol2 = tol * tol;
  set_status_kernel<<<cdiv(R, 256), 256, 0, st>>>(R, w.sc.status, w.sc.iters, w.sc.done, w.sc.want,
                                                   w.sc.rz, d_mask);
  // |b|^2 and the stopping thresholds
  dot_partial_kernel<T><<<L.grid, L.block, L.smem, st>>>(S.n, R, w.Rv, w.Rv, w.part);
  reduce_kernel<<<1, 1024, 0, st>>>(nblk2, R, w.part, RED_INIT_B, w.sc, nullptr);
  if (d_b2ref) set_thresholds_kernel<<<cdiv(R, 256), 256, 0, st>>>(R, w.sc.tol2, d_b2ref, w.sc);
  MBC_CK(cudaMemsetAsync(w.Pv, 0, sizeof(T) * (size_t)S.n * R, st));
  MBC_CKL();
  S.launches += (d_b2ref ? 4 : 3);
  int32_t *h_flags = S.h_flag;  // [done, want]
  if (S.profile) MBC_TRY(S.ensure_events(2 * check_every));
  int replaced = 0;
  // Column compaction (compact, no replacement, x of the iteration's own
  // type): once at most half of the current columns are still active, their
  // state moves to a narrower block (ping-pong between two buffer sets) and
  // the iteration continues on it; the stopped columns' x and outcome go back
  // to the caller's arrays then, the rest at the end.  `cols` maps current
  // columns to the caller's.
  compact = compact && !replace && std::is_same<T, XT>::value;
  PcgWork<T> *cw = &w;
  XT *cx = x;
  int cR = R;
  Layout2D cL = L;
  int cnblk2 = nblk2;
  PcgWork<T> wc[2];
  DevMem cwork[2], cpart[2], cscal[2], cidx;
  int flip = 0;
  bool compacted = false;
  std::vector<int32_t> cols;
  auto save_to_caller = [&]() -> mbc_status {
    // every current column's x and outcome into the caller's arrays
    MBC_TRY(cidx.reserve(sizeof(int32_t) * (size_t)R));
    int32_t *d_cols = (int32_t *)cidx.ptr;
    MBC_CK(cudaMemcpyAsync(d_cols, cols.data(), sizeof(int32_t) * cR, cudaMemcpyHostToDevice, st));
    scatter_scalars_kernel<<<cdiv(cR, 256), 256, 0, st>>>(cR, d_cols, cw->sc, w.sc);
    const int64_t ns = (int64_t)S.n * cR;
    scatter_cols_kernel<XT><<<cdiv(ns, 256), 256, 0, st>>>(S.n, R, cR, d_cols, cx, x);
    S.launches += 2;
    MBC_CKL();
    return MBC_OK;
  };
  for (int it = 0; it < maxit; it += check_every) {
    const int kmax = std::min(check_every, maxit - it);
    // (the captured block holds kernel launches only: the unpreconditioned
    // variant's checked copy and the profiling events stay eager)
    const bool use_graph = S.graph && precond && !S.profile && it > 0 && kmax == check_every;
    if (use_graph && graph.exec) {
      MBC_CK(cudaGraphLaunch(graph.exec, st));
      S.launches += graph_launches;
    }
    const int64_t launches_before = S.launches;
    if (use_graph && !graph.exec) MBC_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
    for (int k = 0; k < kmax && !(use_graph && graph.exec && graph_launches > 0); ++k) {
      if (precond) {
        precond_lt_kernel<T, LT><<<cL.grid, cL.block, 0, st>>>(S.n, cR, S.d_lptr(), S.d_lind(), lval,
                                                                cw->Rv, cw->U, cw->sc.done);
        precond_l_kernel<T, LT><<<cL.grid, cL.block, cL.smem, st>>>(S.n, cR, S.d_rptr(), S.d_rcol(),
                                                                   S.d_rmap(), lval, cw->U, cw->Z, cw->Rv,
                                                                   cw->part, cw->sc.done);
      } else {
        MBC_CK(cudaMemcpyAsync(cw->Z, cw->Rv, sizeof(T) * (size_t)S.n * cR, cudaMemcpyDeviceToDevice, st));
        dot_partial_kernel<T><<<cL.grid, cL.block, cL.smem, st>>>(S.n, cR, cw->Rv, cw->Z, cw->part);
      }
      reduce_kernel<<<1, 1024, 0, st>>>(cnblk2, cR, cw->part, RED_BETA, cw->sc, nullptr);
      update_p_kernel<T><<<cL.grid, cL.block, 0, st>>>(S.n, cR, cw->sc.beta, cw->sc.status, cw->Z, cw->Pv,
                                                        cw->sc.done);
      if (S.profile) MBC_CK(cudaEventRecord(S.events[2 * k], st));
      launch_rows<T>(S, cR, cw->Pv, cw->W, cw->sc.done, st);
      const int nb = launch_cols<T>(S, cR, cw->W, cw->Tt, cw->Pv, cw->part, cw->sc.done, st);
      if (S.profile) MBC_CK(cudaEventRecord(S.events[2 * k + 1], st));
      reduce_kernel<<<1, 1024, 0, st>>>(nb, cR, cw->part, RED_ALPHA, cw->sc, nullptr);
      update_xr_kernel<T, XT><<<cL.grid, cL.block, cL.smem, st>>>(S.n, cR, cw->sc.alpha, cw->Pv, cw->Tt, cx,
                                                                 cw->Rv, cw->part, cw->sc.done);
      reduce_kernel<<<1, 1024, 0, st>>>(cnblk2, cR, cw->part, RED_CHECK, cw->sc, nullptr);
      S.launches += precond ? 7 : 6;  // the matvec pair counts itself
    }
    if (use_graph && !graph.exec) {
      cudaGraph_t g = nullptr;
      const cudaError_t ec = cudaStreamEndCapture(st, &g);
      if (ec != cudaSuccess) return fail(MBC_CUDA_ERROR, std::string("capture of a PCG block: ") + cudaGetErrorString(ec));
      const cudaError_t ei = cudaGraphInstantiate(&graph.exec, g, 0);
      cudaGraphDestroy(g);
      if (ei != cudaSuccess) return fail(MBC_CUDA_ERROR, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ei));
      graph_launches = S.launches - launches_before;
      MBC_CK(cudaGraphLaunch(graph.exec, st));
    }
    MBC_CKL();
    MBC_CK(cudaMemcpyAsync(h_flags, cw->sc.done, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    MBC_CK(cudaStreamSynchronize(st));
    if (S.profile) {
      // iterations after the last active column stopped exit at once; they
      // are filtered out when the stats are formed
      for (int k = 0; k < kmax; ++k) {
        float ms = 0.f;
        MBC_CK(cudaEventElapsedTime(&ms, S.events[2 * k], S.events[2 * k + 1]));
        S.prof_ms_all.push_back(ms);
        S.prof_is64.push_back(sizeof(T) == 8 ? 1 : 0);
        S.prof_cols.push_back(cR);
      }
    }
    if (h_flags[0]) break;
    if (replace && h_flags[1] && replaced < max_replace) {
      MBC_TRY((*replace)());
      ++replaced;
      MBC_CK(cudaMemsetAsync(w.sc.want, 0, sizeof(int32_t), st));
      MBC_CK(cudaMemcpyAsync(h_flags, w.sc.done, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
      MBC_CK(cudaStreamSynchronize(st));
      if (h_flags[0]) break;
    }
    if constexpr (std::is_same<T, XT>::value) {
      if (compact && it + check_every < maxit) {
        std::vector<int32_t> stat(cR);
        MBC_CK(cudaMemcpyAsync(stat.data(), cw->sc.status, sizeof(int32_t) * cR, cudaMemcpyDeviceToHost, st));
        MBC_CK(cudaStreamSynchronize(st));
        std::vector<int32_t> act;
        for (int c = 0; c < cR; ++c)
          if (stat[c] == COL_ACTIVE) act.push_back(c);
        const int A = (int)act.size();
        if (A > 0 && 2 * A <= cR && cR - A >= 8) {
          if (!compacted) {
            cols.resize(R);
            for (int c = 0; c < R; ++c) cols[c] = c;
          } else {
            MBC_TRY(save_to_caller());
          }
          PcgWork<T> &nw = wc[flip];
          MBC_TRY(pcg_buffers_in<T>(S, A, nw, cwork[flip], cpart[flip], cscal[flip]));
          MBC_TRY(cidx.reserve(sizeof(int32_t) * (size_t)R));
          int32_t *d_act = (int32_t *)cidx.ptr;
          MBC_CK(cudaMemcpyAsync(d_act, act.data(), sizeof(int32_t) * A, cudaMemcpyHostToDevice, st));
          const int64_t ns = (int64_t)S.n * A;
          gather_cols_kernel<T><<<cdiv(ns, 256), 256, 0, st>>>(S.n, cR, A, d_act, cx, nw.X);
          gather_cols_kernel<T><<<cdiv(ns, 256), 256, 0, st>>>(S.n, cR, A, d_act, cw->Rv, nw.Rv);
          gather_cols_kernel<T><<<cdiv(ns, 256), 256, 0, st>>>(S.n, cR, A, d_act, cw->Pv, nw.Pv);
          gather_scalars_kernel<<<cdiv(A, 256), 256, 0, st>>>(A, d_act, cw->sc, nw.sc);
          S.launches += 4;
          MBC_CKL();
          nw.sc.maxit = cw->sc.maxit;
          nw.sc.tol2 = cw->sc.tol2;
          nw.sc.drop2 = cw->sc.drop2;
          std::vector<int32_t> ncols(A);
          for (int k = 0; k < A; ++k) ncols[k] = cols[act[k]];
          cols.swap(ncols);
          // the next block waits for the gathers (same stream); the source
          // buffers are not touched again
          MBC_CK(cudaStreamSynchronize(st));
          cw = &nw;
          cx = nw.X;
          cR = A;
          cL = layout2d(S.n, A);
          cnblk2 = (int)cL.grid.x;
          flip ^= 1;
          compacted = true;
          if (graph.exec) {  // the captured block has the old width baked in
            cudaGraphExecDestroy(graph.exec);
            graph.exec = nullptr;
            graph_launches = 0;
          }
        }
      }
    }
  }
  if (compacted) MBC_TRY(save_to_caller());
  S.replacements = replaced;
  return MBC_OK;
}

// Block PCG: the outcome of one step for the active columns act[0 .. a) of
// the caller's batch: rr = |r|^2 (FP64), iteration count, converge / max
// iterations / breakdown (NaN) tests against each column's threshold.
__global__ void block_check_kernel(int a, const int32_t *__restrict__ act, const double *__restrict__ rr,
                                   PcgScalars sc)
{
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a) return;
  const int c = act[j];
  if (sc.status[c] != COL_ACTIVE) return;
  const double s = rr[j];
  sc.rr[c] = s;
  sc.iters[c] += 1;
  if (!(s == s)) sc.status[c] = COL_BREAKDOWN;
  else if (s < sc.thr[c]) sc.status[c] = COL_OK;
  else if (sc.iters[c] >= sc.maxit) sc.status[c] = COL_MAXIT;
}

// every column in act[0 .. a) still active gets status `st` (a breakdown of the block step)
__global__ void block_fail_kernel(int a, const int32_t *__restrict__ act, PcgScalars sc, int32_t st)
{
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < a && sc.status[act[j]] == COL_ACTIVE) sc.status[act[j]] = st;
}

// Block PCG on (K^T K) X = B for R columns (schedule MBC_SCHED_BLOCK):
// O'Leary's block conjugate gradients with the KL preconditioner, search
// blocks kept orthonormal (rank-revealing Cholesky QR, one pass; block.cuh).
// All active columns share one Krylov space, so a column whose own Krylov
// space converges slowly is helped by the directions the other columns
// found.  One step, for the active columns (compact, n x a):
//   Q = A P;  G = P^T Q;  alpha = G^-1 P^T R;  X += P alpha;  R -= Q alpha;
//   per-column stop test on |r|^2 (the thresholds of the batched PCG);
//   Z = M R (still active columns);  beta = -G^-1 Q^T Z;
//   P = orth(Z + P beta).
// Columns leave the block as they converge (their X goes back to w.X), so
// the matvec and the dense products shrink with the active set.  On entry
// w.X holds x0 and w.Rv the residual b - A x0 (new order, n x R); on exit
// w.X holds the solutions and w.sc the per-column status, iterations and
// |r|^2.  FP64 throughout (the matvec per the solver's FP64 choice).
// columns the block PCG keeps while any column iterates.  Narrow INT8
// matvecs are bound by the digit-plane stream, so a wider tail block costs
// little: at N = 64000 one launch takes 3.4 ms at 16 columns and 4.1 ms at
// 48.  Measured on the 32-ellipsoid trajectory (8 poses, B200): 48 gives 4.6 %
// fewer column-iterations and 2.5 % shorter steps than 16; 64 and 96 lower
// the iterations further but lengthen the steps.
constexpr int kBlockKeep = 48;

template <typename LT>
static mbc_status run_block_pcg(Solver &S, int R, PcgWork<double> &w, const LT *lval, int maxit, double tol,
                                const double *d_b2ref, cudaStream_t st)
{
  const int n = S.n;
  if (R > blk::kOrthMax) return fail(MBC_UNSUPPORTED, "block PCG: more than 512 columns");
  const Layout2D L0 = layout2d(n, R);
  w.sc.maxit = maxit;
  w.sc.tol2 = tol * tol;
  set_status_kernel<<<cdiv(R, 256), 256, 0, st>>>(R, w.sc.status, w.sc.iters, w.sc.done, w.sc.want, w.sc.rz,
                                                   nullptr);
  dot_partial_kernel<double><<<L0.grid, L0.block, L0.smem, st>>>(n, R, w.Rv, w.Rv, w.part);
  reduce_kernel<<<1, 1024, 0, st>>>((int)L0.grid.x, R, w.part, RED_INIT_B, w.sc, nullptr);
  if (d_b2ref) set_thresholds_kernel<<<cdiv(R, 256), 256, 0, st>>>(R, w.sc.tol2, d_b2ref, w.sc);
  S.launches += d_b2ref ? 4 : 3;
  MBC_CKL();
  // device memory: compact X / R (two sets), search blocks P and V, small
  // matrices (ld R), Gram partials, index lists
  const size_t nv = (size_t)n * R, sm = (size_t)R * R;
  const int chunks = blk::gram_chunks(n);
  const size_t bytes = sizeof(double) * (6 * nv + 6 * sm + (size_t)chunks * sm + 2 * R) + sizeof(int32_t) * (3 * R + 8);
  MBC_TRY(S.blk.reserve(bytes));
  double *base = (double *)S.blk.ptr;
  double *Xa[2] = {base, base + nv}, *Ra[2] = {base + 2 * nv, base + 3 * nv};
  double *P = base + 4 * nv, *V = base + 5 * nv;
  double *G = base + 6 * nv, *Sm = G + sm, *H = Sm + sm, *Wm = H + sm, *T1 = Wm + sm, *T2 = T1 + sm;
  double *gpart = T2 + sm, *rr = gpart + (size_t)chunks * sm, *oscale = rr + R;
  int32_t *d_act = (int32_t *)(oscale + R), *d_loc = d_act + R, *d_perm = d_loc + R, *d_small = d_perm + R;
  double *Q = w.Tt, *Z = w.Z, *U = w.U, *W = w.W;
  // host view
  std::vector<int32_t> status(R), act, loc;
  int32_t *h_small = S.h_flag;  // pinned: [rank, flag]
  auto gram = [&](const double *A, int lda, int ka, const double *B, int ldb, int kb, double *C) {
    const dim3 g((unsigned)chunks, cdiv(ka, blk::kTile), cdiv(kb, blk::kTile));
    blk::gram_partial_kernel<<<g, blk::kThreads, 0, st>>>(n, A, lda, ka, B, ldb, kb, gpart);
    blk::gram_reduce_kernel<<<cdiv((int64_t)ka * kb, 256), 256, 0, st>>>(chunks, ka, kb, gpart, C, R);
    S.launches += 2;
  };
  auto update = [&](int k, int m, const double *Pm, int ldp, const double *M, const double *bse, int ldb,
                    double sgn, double *out, int ldo, const int32_t *skip = nullptr) {
    const dim3 g(cdiv(n, blk::kTile), cdiv(m, blk::kTile));
    blk::block_update_kernel<<<g, blk::kThreads, 0, st>>>(n, k, m, Pm, ldp, M, R, bse, ldb, sgn, out, ldo, skip);
    ++S.launches;
  };
  auto precond = [&](int a, const double *Rm, double *Zm) {
    const Layout2D La = layout2d(n, a);
    precond_lt_kernel<double, LT><<<La.grid, La.block, 0, st>>>(n, a, S.d_lptr(), S.d_lind(), lval, Rm, U, nullptr);
    precond_l_kernel<double, LT><<<La.grid, La.block, La.smem, st>>>(n, a, S.d_rptr(), S.d_rcol(), S.d_rmap(), lval,
                                                                      U, Zm, Rm, w.part, nullptr);
    S.launches += 2;
  };
  // the small factorizations keep their matrix's lower triangle in shared
  // memory (packed) when it fits; the column-parallel solves add one column
  // per warp
  auto packed = [](int k) -> int { return k <= blk::kPackedDim; };
  auto smem_fac = [&](int k) -> size_t { return packed(k) ? sizeof(double) * blk::packed_len(k) : 0; };
  auto smem_sol = [&](int k) -> size_t { return sizeof(double) * (size_t)blk::kSolveWarps * k + smem_fac(k); };
  const size_t smem_sol_max = std::max(smem_sol(blk::kPackedDim), smem_sol(blk::kOrthMax));
  MBC_TRY(allow_max_smem(blk::chol_kernel, smem_fac(blk::kPackedDim)));
  MBC_TRY(allow_max_smem(blk::orth_factor_kernel, smem_fac(blk::kPackedDim)));
  MBC_TRY(allow_max_smem(blk::chol_solve_kernel, smem_sol_max));
  MBC_TRY(allow_max_smem(blk::orth_t_kernel, smem_sol_max));
  // P (n x r, ld r) = an orthonormal basis of the columns of Vin (n x m, ld
  // m; Vin is P's partner buffer V or Z, not needed afterwards), dependent
  // directions dropped; r = 0 when none is left.  One Cholesky QR pass: the
  // drop bounds the kept block's condition by ~1e6, so P's orthogonality
  // error, of order eps cond^2 <= 1e-4, leaves P^T A P well conditioned,
  // which is all the recursion needs (it never assumes P^T P = I).
  auto orth = [&](const double *Vin, int m, int *r_out) -> mbc_status {
    gram(Vin, m, m, Vin, m, m, Wm);
    blk::orth_factor_kernel<<<1, blk::kSmallThreads, smem_fac(m), st>>>(m, Wm, R, 1e-6, oscale, d_perm, d_small,
                                                                         packed(m));
    blk::orth_t_kernel<<<cdiv(m, blk::kSolveWarps), blk::kSolveWarps * 32, smem_sol(m), st>>>(
        m, Wm, R, oscale, d_perm, d_small, T1, R, packed(m));
    MBC_CK(cudaMemcpyAsync(h_small, d_small, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    MBC_CK(cudaStreamSynchronize(st));
    const int r = h_small[0];
    S.launches += 2;
    *r_out = r;
    if (r > 0) update(m, r, Vin, m, T1, nullptr, 0, 1.0, P, r);
    return MBC_OK;
  };
  // the active columns, gathered into the compact block
  MBC_CK(cudaMemcpyAsync(status.data(), w.sc.status, sizeof(int32_t) * R, cudaMemcpyDeviceToHost, st));
  MBC_CK(cudaStreamSynchronize(st));
  for (int c = 0; c < R; ++c)
    if (status[c] == COL_ACTIVE) act.push_back(c);
  int a = (int)act.size();
  if (a == 0) return MBC_OK;
  int cur = 0;
  MBC_CK(cudaMemcpyAsync(d_act, act.data(), sizeof(int32_t) * a, cudaMemcpyHostToDevice, st));
  gather_cols_kernel<double><<<cdiv((int64_t)n * a, 256), 256, 0, st>>>(n, R, a, d_act, w.X, Xa[cur]);
  gather_cols_kernel<double><<<cdiv((int64_t)n * a, 256), 256, 0, st>>>(n, R, a, d_act, w.Rv, Ra[cur]);
  S.launches += 2;
  precond(a, Ra[cur], Z);
  int k = 0;
  MBC_TRY(orth(Z, a, &k));
  if (S.profile) MBC_TRY(S.ensure_events(2));
  int32_t *d_flag = d_small + 1;
  bool failed = false;
  for (int it = 0; it < maxit && k > 0; ++it) {
    if (S.profile) MBC_CK(cudaEventRecord(S.events[0], st));
    launch_rows<double>(S, k, P, W, nullptr, st);
    launch_cols<double>(S, k, W, Q, nullptr, nullptr, nullptr, st);
    if (S.profile) MBC_CK(cudaEventRecord(S.events[1], st));
    // alpha = (P^T A P)^-1 P^T R;  X += P alpha;  R -= Q alpha
    gram(P, k, k, Q, k, k, G);
    gram(P, k, k, Ra[cur], a, a, Sm);
    MBC_CK(cudaMemsetAsync(d_flag, 0, sizeof(int32_t), st));
    blk::chol_kernel<<<1, blk::kSmallThreads, smem_fac(k), st>>>(k, G, R, d_flag, packed(k));
    blk::chol_solve_kernel<<<cdiv(a, blk::kSolveWarps), blk::kSolveWarps * 32, smem_sol(k), st>>>(
        k, G, R, a, Sm, R, 1.0, d_flag, packed(k));
    update(k, a, P, k, Sm, Xa[cur], a, 1.0, Xa[cur], a, d_flag);
    update(k, a, Q, k, Sm, Ra[cur], a, -1.0, Ra[cur], a, d_flag);
    // per-column stop test on |r|^2
    const Layout2D La = layout2d(n, a);
    dot_partial_kernel<double><<<La.grid, La.block, La.smem, st>>>(n, a, Ra[cur], Ra[cur], w.part);
    PcgScalars none{};
    reduce_kernel<<<1, 1024, 0, st>>>((int)La.grid.x, a, w.part, RED_STORE, none, rr);
    block_check_kernel<<<cdiv(a, 256), 256, 0, st>>>(a, d_act, rr, w.sc);
    S.launches += 6;
    MBC_CKL();
    MBC_CK(cudaMemcpyAsync(status.data(), w.sc.status, sizeof(int32_t) * R, cudaMemcpyDeviceToHost, st));
    MBC_CK(cudaMemcpyAsync(h_small + 1, d_flag, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    MBC_CK(cudaStreamSynchronize(st));
    if (S.profile) {
      float ms = 0.f;
      MBC_CK(cudaEventElapsedTime(&ms, S.events[0], S.events[1]));
      S.prof_ms_all.push_back(ms);
      S.prof_is64.push_back(1);
      S.prof_cols.push_back(k);
    }
    if (h_small[1]) {  // P^T A P not positive definite (NaN or breakdown): nothing was updated
      failed = true;
      break;
    }
    std::vector<int32_t> keep;  // positions in the compact block of the columns still active
    for (int j = 0; j < a; ++j)
      if (status[act[j]] == COL_ACTIVE) keep.push_back(j);
    const int nact = (int)keep.size();
    // While any column iterates, the block keeps at least kBlockKeep columns:
    // converged ones stay in (their x keeps improving; their stop state is
    // final) and go on feeding the shared Krylov space with directions, at
    // little matvec cost (above).  The slowest columns' tail is where this
    // pays.
    if (nact > 0 && nact < std::min(a, kBlockKeep)) {
      std::vector<char> in(a, 0);
      for (int j : keep) in[j] = 1;
      for (int j = a - 1; j >= 0 && (int)keep.size() < std::min(a, kBlockKeep); --j)
        if (!in[j]) keep.push_back(j);
      std::sort(keep.begin(), keep.end());
    }
    const int a2 = nact == 0 ? 0 : (int)keep.size();
    if (a2 < a) {
      // finished columns' x back to the batch (the others are rewritten later)
      scatter_cols_kernel<double><<<cdiv((int64_t)n * a, 256), 256, 0, st>>>(n, R, a, d_act, Xa[cur], w.X);
      ++S.launches;
      if (a2 == 0) {
        a = 0;
        break;
      }
      MBC_CK(cudaMemcpyAsync(d_loc, keep.data(), sizeof(int32_t) * a2, cudaMemcpyHostToDevice, st));
      gather_cols_kernel<double><<<cdiv((int64_t)n * a2, 256), 256, 0, st>>>(n, a, a2, d_loc, Xa[cur], Xa[cur ^ 1]);
      gather_cols_kernel<double><<<cdiv((int64_t)n * a2, 256), 256, 0, st>>>(n, a, a2, d_loc, Ra[cur], Ra[cur ^ 1]);
      S.launches += 2;
      std::vector<int32_t> act2(a2);
      for (int j = 0; j < a2; ++j) act2[j] = act[keep[j]];
      act.swap(act2);
      MBC_CK(cudaMemcpyAsync(d_act, act.data(), sizeof(int32_t) * a2, cudaMemcpyHostToDevice, st));
      cur ^= 1;
      a = a2;
    }
    // next search block: P = orth(Z + P beta), beta = -(P^T A P)^-1 Q^T Z
    precond(a, Ra[cur], Z);
    gram(Q, k, k, Z, a, a, H);
    blk::chol_solve_kernel<<<cdiv(a, blk::kSolveWarps), blk::kSolveWarps * 32, smem_sol(k), st>>>(
        k, G, R, a, H, R, -1.0, nullptr, packed(k));
    update(k, a, P, k, H, Z, a, 1.0, V, a);
    S.launches += 1;
    MBC_TRY(orth(V, a, &k));
  }
  if (a > 0) {
    // out of iterations, no search direction left, or a failed step: the
    // columns still active end as not converged (their x as it stands)
    scatter_cols_kernel<double><<<cdiv((int64_t)n * a, 256), 256, 0, st>>>(n, R, a, d_act, Xa[cur], w.X);
    block_fail_kernel<<<cdiv(a, 256), 256, 0, st>>>(a, d_act, w.sc, COL_MAXIT);
    S.launches += 2;
    MBC_CKL();
  }
  (void)failed;
  return MBC_OK;
}

// residual r = K^T (f - K x) in T, all columns; f, x new-order buffers
template <typename T>
static void residual(Solver &S, int R, const T *F, const T *X, T *W, T *Rout, cudaStream_t st)
{
  launch_rows<T>(S, R, X, W, nullptr, st);
  const int64_t cnt = (int64_t)S.nf * R;
  sub_kernel<T><<<cdiv(cnt, 256), 256, 0, st>>>(cnt, F, W, W);
  launch_cols<T>(S, R, W, Rout, nullptr, nullptr, nullptr, st);
  ++S.launches;
}

// per-column norms^2 of an n x R array into host vector
template <typename T>
static mbc_status col_norms2(Solver &S, int R, const T *A, std::vector<double> &out, cudaStream_t st)
{
  const Layout2D L = layout2d(S.n, R);
  // own buffer: S.part may be referenced by a live PcgWork
  MBC_TRY(S.nrm.reserve(sizeof(double) * ((size_t)L.grid.x * R + R)));
  double *part = (double *)S.nrm.ptr;
  double *res = part + (size_t)L.grid.x * R;
  dot_partial_kernel<T><<<L.grid, L.block, L.smem, st>>>(S.n, R, A, A, part);
  PcgScalars sc{};
  reduce_kernel<<<1, 1024, 0, st>>>((int)L.grid.x, R, part, RED_STORE, sc, res);
  S.launches += 2;
  MBC_CKL();
  out.resize(R);
  MBC_CK(cudaMemcpyAsync(out.data(), res, sizeof(double) * R, cudaMemcpyDeviceToHost, st));
  MBC_CK(cudaStreamSynchronize(st));
  return MBC_OK;
}

// per-column norms^2 of an n x R array into a device vector (R doubles)
template <typename T>
static mbc_status col_norms2_dev(Solver &S, int R, const T *A, double *out, cudaStream_t st)
{
  const Layout2D L = layout2d(S.n, R);
  MBC_TRY(S.nrm.reserve(sizeof(double) * (size_t)L.grid.x * R));
  double *part = (double *)S.nrm.ptr;
  dot_partial_kernel<T><<<L.grid, L.block, L.smem, st>>>(S.n, R, A, A, part);
  PcgScalars sc{};
  reduce_kernel<<<1, 1024, 0, st>>>((int)L.grid.x, R, part, RED_STORE, sc, out);
  S.launches += 2;
  MBC_CKL();
  return MBC_OK;
}

template <typename S_, typename D_>
static void convert(int64_t cnt, const S_ *a, D_ *b, cudaStream_t st)
{
  convert_kernel<S_, D_><<<cdiv(cnt, 256), 256, 0, st>>>(cnt, a, b);
}

template <typename D_>
static void permute_in(Solver &S, int R, const void *src, int32_t dt, D_ *dst, cudaStream_t st)
{
  const int64_t cnt = (int64_t)S.n * R;
  ++S.launches;
  if (dt == MBC_F64)
    permute_in_kernel<double, D_><<<cdiv(cnt, 256), 256, 0, st>>>(S.n, R, S.dP(), (const double *)src, dst);
  else
    permute_in_kernel<float, D_><<<cdiv(cnt, 256), 256, 0, st>>>(S.n, R, S.dP(), (const float *)src, dst);
}

template <typename S_>
static void permute_out(Solver &S, int R, const S_ *src, void *dst, int32_t dt, cudaStream_t st)
{
  const int64_t cnt = (int64_t)S.n * R;
  ++S.launches;
  if (dt == MBC_F64)
    permute_out_kernel<S_, double><<<cdiv(cnt, 256), 256, 0, st>>>(S.n, R, S.dP(), src, (double *)dst);
  else
    permute_out_kernel<S_, float><<<cdiv(cnt, 256), 256, 0, st>>>(S.n, R, S.dP(), src, (float *)dst);
}

template <typename D_>
static void load_rows(Solver &S, int R, const void *src, int32_t dt, D_ *dst, cudaStream_t st)
{
  const int64_t cnt = (int64_t)S.nf * R;
  ++S.launches;
  if (dt == MBC_F64) convert<double, D_>(cnt, (const double *)src, dst, st);
  else convert<float, D_>(cnt, (const float *)src, dst, st);
}

// Collect per-column results of the last run_pcg into stats.
template <typename T>
static mbc_status collect(Solver &S, int R, PcgWork<T> &w, std::vector<int32_t> &status,
                          std::vector<int32_t> &iters, std::vector<double> &rel, cudaStream_t st)
{
  std::vector<double> rr(R), b2(R);
  status.resize(R);
  iters.resize(R);
  MBC_CK(cudaMemcpyAsync(status.data(), w.sc.status, sizeof(int32_t) * R, cudaMemcpyDeviceToHost, st));
  MBC_CK(cudaMemcpyAsync(iters.data(), w.sc.iters, sizeof(int32_t) * R, cudaMemcpyDeviceToHost, st));
  MBC_CK(cudaMemcpyAsync(rr.data(), w.sc.rr, sizeof(double) * R, cudaMemcpyDeviceToHost, st));
  MBC_CK(cudaMemcpyAsync(b2.data(), w.sc.b2, sizeof(double) * R, cudaMemcpyDeviceToHost, st));
  MBC_CK(cudaStreamSynchronize(st));
  rel.resize(R);
  for (int c = 0; c < R; ++c) rel[c] = b2[c] < 1e-16 ? 0.0 : std::sqrt(rr[c] / b2[c]);
  return MBC_OK;
}

static mbc_status finish_stats(int R, const std::vector<int32_t> &status, const std::vector<int32_t> &iters,
                               const std::vector<double> &rel, mbc_solve_stats *st_out,
                               int32_t *iters_host)
{
  mbc_solve_stats s{};
  s.true_relres_max = -1;
  int worst = 0;
  for (int c = 0; c < R; ++c) {
    s.iters_max = std::max(s.iters_max, iters[c]);
    s.iters_total += iters[c];
    if (status[c] == COL_OK) ++s.n_converged;
    s.relres_max = std::max(s.relres_max, rel[c]);
    int code = status[c] == COL_OK ? 0 : status[c] == COL_BREAKDOWN ? 2 : 1;
    worst = std::max(worst, code);
    if (iters_host) iters_host[c] = iters[c];
  }
  s.status_per_worst = worst;
  if (st_out) *st_out = s;
  return MBC_OK;
}

// Plain (MBC_F64) or reference-style single-sweep solve in precision T.
// mode 0: forward with F; mode 1: adjoint with B.
template <typename T>
mbc_status Solver::solve_plain(int R, const void *rhs, int32_t rhs_dt, void *X, int32_t x_dt,
                               const void *X0, bool adjoint, const mbc_solve_options &o,
                               mbc_solve_stats *stats, int32_t *iters_host, cudaStream_t st)
{
  PcgWork<T> w;
  MBC_TRY(pcg_buffers<T>(*this, R, w));
  // F (forward) lives in fbuf (T, nf x R); with the INT8 FP64 operator the
  // adjoint right-hand side b is kept there too (n x R), for the residual
  // checks after the PCG
  DevMem &fm = sizeof(T) == 8 ? fbuf64 : fbuf32;
  const bool oz = sizeof(T) == 8 && use_oz(*this);
  if (!adjoint) {
    MBC_TRY(fm.reserve(sizeof(T) * (size_t)nf * R));
    load_rows<T>(*this, R, rhs, rhs_dt, (T *)fm.ptr, st);
  } else if (oz) {
    MBC_TRY(fm.reserve(sizeof(T) * (size_t)n * R));
    permute_in<T>(*this, R, rhs, rhs_dt, (T *)fm.ptr, st);
  }
  const int64_t nv = (int64_t)n * R;
  if (X0) {
    permute_in<T>(*this, R, X0, x_dt, w.X, st);
    if (adjoint) {
      // r = b - K^T K x0
      permute_in<T>(*this, R, rhs, rhs_dt, w.Z, st);
      launch_rows<T>(*this, R, w.X, w.W, nullptr, st);
      launch_cols<T>(*this, R, w.W, w.Tt, nullptr, nullptr, nullptr, st);
      sub_kernel<T><<<cdiv(nv, 256), 256, 0, st>>>(nv, w.Z, w.Tt, w.Rv);
    } else {
      residual<T>(*this, R, (const T *)fm.ptr, w.X, w.W, w.Rv, st);
    }
  } else {
    MBC_CK(cudaMemsetAsync(w.X, 0, sizeof(T) * nv, st));
    if (adjoint) permute_in<T>(*this, R, rhs, rhs_dt, w.Rv, st);
    else launch_cols<T>(*this, R, (const T *)fm.ptr, w.Rv, nullptr, nullptr, nullptr, st);
  }
  MBC_CKL();
  // A warm start keeps the thresholds relative to |b| (b = K^T f or the adjoint rhs).
  const double *b2 = nullptr;
  if (X0) {
    MBC_TRY(b2ref.reserve(sizeof(double) * R));
    T *bvec = w.Tt;
    if (adjoint) permute_in<T>(*this, R, rhs, rhs_dt, bvec, st);
    else launch_cols<T>(*this, R, (const T *)fm.ptr, bvec, nullptr, nullptr, nullptr, st);
    MBC_TRY(col_norms2_dev<T>(*this, R, bvec, (double *)b2ref.ptr, st));
    b2 = (const double *)b2ref.ptr;
  }
  const bool compact = o.compact != 0;
  // block PCG (FP64 recursions only; the preconditioner is always applied)
  const bool block = sizeof(T) == 8 && o.schedule == MBC_SCHED_BLOCK && R > 1;
  // With the INT8 operator the recursion's own residual drifts from the
  // FP64 one by up to ~20 % near tol (measured at N = 64000): its columns run
  // to 0.85 tol, so that few fail the FP64 decision below and restart.
  const double rtol = oz ? 0.85 * o.tol : o.tol;
  if (block) {
    if constexpr (sizeof(T) == 8) {
      PcgWork<double> &wd = reinterpret_cast<PcgWork<double> &>(w);
      if (precision == MBC_F64)
        MBC_TRY(run_block_pcg<double>(*this, R, wd, (const double *)lval.ptr, o.max_iters, rtol, b2, st));
      else
        MBC_TRY(run_block_pcg<float>(*this, R, wd, (const float *)lval.ptr, o.max_iters, rtol, b2, st));
    }
  } else if (precision == MBC_F64) {
    MBC_TRY((run_pcg<T, double, T>(*this, R, w, w.X, (const double *)lval.ptr, o.max_iters, rtol,
                                   o.precondition != 0, std::max(1, o.check_every), nullptr, st, b2,
                                   nullptr, 0, compact)));
  } else {
    MBC_TRY((run_pcg<T, float, T>(*this, R, w, w.X, (const float *)lval.ptr, o.max_iters, rtol,
                                  o.precondition != 0, std::max(1, o.check_every), nullptr, st, b2,
                                  nullptr, 0, compact)));
  }
  std::vector<int32_t> status, iters;
  std::vector<double> rel;
  MBC_TRY(collect<T>(*this, R, w, status, iters, rel, st));
  if constexpr (sizeof(T) == 8) {
    if (oz || block) {
      // The INT8 FP64 operator carries a ~1e-9 relative error (measured on
      // the B200 at the solution), and the block recursion's residual drifts
      // further from the true one than a single column's, so the recursive
      // residual can end above tol once recomputed.  Every column is decided
      // on its residual recomputed with the solver's operator, and those
      // above the threshold restart (batched per-column PCG) from where they
      // stand, at most twice.  A restart builds a fresh Krylov space from the
      // accurate residual; replacing the residual inside the recursion
      // instead stalls the ill-conditioned columns (measured: 544 against 179
      // iterations on one column of a 3000-point scene).
      // The decision residual is FP64-accurate: the products whose inputs
      // cancel against the right-hand side (K x for the forward residual
      // f - K x, both products of the adjoint's b - K^T K x) run on the FP64
      // CUDA-core kernels.  K x of the solution carries the INT8 operator's
      // ~1e-9 relative error against a least-squares residual f - K x ~1e-7
      // |f|; K^T of that residual on the INT8 matvec agrees with FP64 to
      // ~10 digits (measured), so it stays there.  Only |b| (a norm) uses
      // the solver's FP64 matvec as it is.
      T *bvec = w.Tt;
      if (adjoint) MBC_CK(cudaMemcpyAsync(bvec, fm.ptr, sizeof(T) * nv, cudaMemcpyDeviceToDevice, st));
      else launch_cols<T>(*this, R, (const T *)fm.ptr, bvec, nullptr, nullptr, nullptr, st);
      MBC_CKL();
      std::vector<double> nb;
      MBC_TRY(col_norms2<T>(*this, R, bvec, nb, st));
      const int32_t impl = fp64_matvec;
      // the decision residual of Rc columns: F (rhs, nf x Rc; adjoint: b,
      // n x Rc), X (n x Rc) -> Rout (n x Rc), with Wc (nf x Rc), Zc (n x Rc)
      auto resid = [&](int Rc, const T *Fc, const T *Xc, T *Wc, T *Zc, T *Rout) {
        fp64_matvec = MBC_FP64_MATVEC_SIMT;
        launch_rows<T>(*this, Rc, Xc, Wc, nullptr, st);
        if (adjoint) {
          launch_cols<T>(*this, Rc, Wc, Zc, nullptr, nullptr, nullptr, st);
          const int64_t cnt = (int64_t)n * Rc;
          sub_kernel<T><<<cdiv(cnt, 256), 256, 0, st>>>(cnt, Fc, Zc, Rout);
          fp64_matvec = impl;
        } else {
          fp64_matvec = impl;
          const int64_t cnt = (int64_t)nf * Rc;
          sub_kernel<T><<<cdiv(cnt, 256), 256, 0, st>>>(cnt, Fc, Wc, Wc);
          launch_cols<T>(*this, Rc, Wc, Rout, nullptr, nullptr, nullptr, st);
        }
        ++launches;
      };
      // every column decided once; the restarted ones then re-decided alone
      resid(R, (const T *)fm.ptr, w.X, w.W, w.Z, w.Rv);
      MBC_CKL();
      std::vector<double> nr;
      MBC_TRY(col_norms2<T>(*this, R, w.Rv, nr, st));
      std::vector<int32_t> pol;
      for (int c = 0; c < R; ++c) {
        rel[c] = nb[c] < 1e-16 ? 0.0 : std::sqrt(nr[c] / nb[c]);
        if (status[c] == COL_BREAKDOWN) continue;
        status[c] = rel[c] <= o.tol ? COL_OK : COL_MAXIT;
        if (status[c] == COL_MAXIT) pol.push_back(c);
      }
      const int frows = adjoint ? n : nf;
      for (int pass = 0; pass < 2 && !pol.empty(); ++pass) {
        const int Rs = (int)pol.size();
        PcgWork<T> ws;
        DevMem wmem, wpart, wscal, widx, fsub;
        MBC_TRY(pcg_buffers_in<T>(*this, Rs, ws, wmem, wpart, wscal));
        const size_t ib = ((sizeof(int32_t) * Rs) + 15) & ~(size_t)15;
        MBC_TRY(widx.reserve(ib + sizeof(double) * Rs));
        MBC_TRY(fsub.reserve(sizeof(T) * (size_t)frows * Rs));
        int32_t *d_idx = (int32_t *)widx.ptr;
        double *d_b2s = (double *)((char *)widx.ptr + ib);
        std::vector<double> b2s(Rs);
        for (int k = 0; k < Rs; ++k) b2s[k] = nb[pol[k]];
        MBC_CK(cudaMemcpyAsync(d_idx, pol.data(), sizeof(int32_t) * Rs, cudaMemcpyHostToDevice, st));
        MBC_CK(cudaMemcpyAsync(d_b2s, b2s.data(), sizeof(double) * Rs, cudaMemcpyHostToDevice, st));
        const int64_t ns = (int64_t)n * Rs;
        gather_cols_kernel<T><<<cdiv(ns, 256), 256, 0, st>>>(n, R, Rs, d_idx, w.X, ws.X);
        gather_cols_kernel<T><<<cdiv(ns, 256), 256, 0, st>>>(n, R, Rs, d_idx, w.Rv, ws.Rv);
        gather_cols_kernel<T><<<cdiv((int64_t)frows * Rs, 256), 256, 0, st>>>(frows, R, Rs, d_idx,
                                                                             (const T *)fm.ptr, (T *)fsub.ptr);
        launches += 3;
        MBC_CKL();
        // the last restart runs on the FP64 CUDA-core matvec: a column the
        // INT8 operator's ~1e-9 product error keeps above tol (near-singular
        // kernels: sources close to a thin body) converges there, at a cost
        // proportional to the few columns left
        const bool last = pass == 1;
        const double ptol = last ? o.tol : rtol;
        if (last) fp64_matvec = MBC_FP64_MATVEC_SIMT;
        mbc_status prs;
        if (precision == MBC_F64)
          prs = run_pcg<T, double, T>(*this, Rs, ws, ws.X, (const double *)lval.ptr, o.max_iters, ptol,
                                      o.precondition != 0, std::max(1, o.check_every), nullptr, st, d_b2s,
                                      nullptr, 0, compact);
        else
          prs = run_pcg<T, float, T>(*this, Rs, ws, ws.X, (const float *)lval.ptr, o.max_iters, ptol,
                                     o.precondition != 0, std::max(1, o.check_every), nullptr, st, d_b2s,
                                     nullptr, 0, compact);
        fp64_matvec = impl;
        MBC_TRY(prs);
        std::vector<int32_t> it2(Rs);
        MBC_CK(cudaMemcpyAsync(it2.data(), ws.sc.iters, sizeof(int32_t) * Rs, cudaMemcpyDeviceToHost, st));
        // the restarted columns' x back, and their own decision residual
        scatter_cols_kernel<T><<<cdiv(ns, 256), 256, 0, st>>>(n, R, Rs, d_idx, ws.X, w.X);
        resid(Rs, (const T *)fsub.ptr, ws.X, ws.W, ws.Z, ws.Rv);
        scatter_cols_kernel<T><<<cdiv(ns, 256), 256, 0, st>>>(n, R, Rs, d_idx, ws.Rv, w.Rv);
        launches += 2;
        MBC_CKL();
        std::vector<double> nrs;
        MBC_TRY(col_norms2<T>(*this, Rs, ws.Rv, nrs, st));
        std::vector<int32_t> again;
        for (int k = 0; k < Rs; ++k) {
          const int c = pol[k];
          iters[c] += it2[k];
          rel[c] = nb[c] < 1e-16 ? 0.0 : std::sqrt(nrs[k] / nb[c]);
          status[c] = rel[c] <= o.tol ? COL_OK : COL_MAXIT;
          if (status[c] == COL_MAXIT) again.push_back(c);
        }
        pol.swap(again);
      }
    }
  }
  permute_out<T>(*this, R, w.X, X, x_dt, st);
  MBC_CKL();
  MBC_TRY(finish_stats(R, status, iters, rel, stats, iters_host));
  if (stats && o.true_residual && !adjoint) {
    // FP64 |K^T (f - K x)| / |K^T f| on the result
    MBC_TRY(true_residual(R, rhs, rhs_dt, X, x_dt, stats, st));
  }
  MBC_CK(cudaStreamSynchronize(st));
  return MBC_OK;
}

// FP64 true residual of a forward solution (original-order X).
mbc_status Solver::true_residual(int R, const void *F, int32_t f_dt, const void *X, int32_t x_dt,
                                 mbc_solve_stats *stats, cudaStream_t st)
{
  // always the FP64 CUDA-core kernels, whatever FP64 matvec the solves use
  struct Restore {
    Solver &S;
    int32_t impl;
    ~Restore() { S.fp64_matvec = impl; }
  } restore{*this, fp64_matvec};
  fp64_matvec = MBC_FP64_MATVEC_SIMT;
  MBC_TRY(fbuf64.reserve(sizeof(double) * (size_t)nf * R));
  MBC_TRY(res64.reserve(sizeof(double) * ((size_t)nf * R + 2 * (size_t)n * R)));
  double *Fd = (double *)fbuf64.ptr;
  double *Wd = (double *)res64.ptr;
  double *Xd = Wd + (size_t)nf * R;
  double *Rd = Xd + (size_t)n * R;
  load_rows<double>(*this, R, F, f_dt, Fd, st);
  permute_in<double>(*this, R, X, x_dt, Xd, st);
  residual<double>(*this, R, Fd, Xd, Wd, Rd, st);
  launch_cols<double>(*this, R, Fd, Xd, nullptr, nullptr, nullptr, st);  // b = K^T f into Xd
  MBC_CKL();
  std::vector<double> nr, nb;
  MBC_TRY(col_norms2<double>(*this, R, Rd, nr, st));
  MBC_TRY(col_norms2<double>(*this, R, Xd, nb, st));
  double m = 0;
  for (int c = 0; c < R; ++c) m = std::max(m, nb[c] < 1e-16 ? 0.0 : std::sqrt(nr[c] / nb[c]));
  stats->true_relres_max = m;
  return MBC_OK;
}

// Mixed precision: one FP32 PCG recursion (FP32 matvec, factor and
// preconditioner; FP64 scalars and dot products) with the solution
// accumulated in FP64 and residual replacement: whenever a column's
// recursive |r|^2 has dropped by inner_tol^2 since the last replacement, or
// reaches the threshold, r is replaced by the FP64 true residual
// K^T (f - K x) (b - K^T K x for the adjoint).  A column converges only on a
// true residual, so tol is met in FP64 terms; the search direction survives
// each replacement, so the Krylov information is not thrown away.
mbc_status Solver::solve_mixed(int R, const void *rhs, int32_t rhs_dt, void *X, int32_t x_dt,
                               const void *X0, bool adjoint, const mbc_solve_options &o,
                               mbc_solve_stats *stats, int32_t *iters_host, cudaStream_t st)
{
  const size_t nv = (size_t)n * R, fv = (size_t)nf * R;
  MBC_TRY(fbuf64.reserve(sizeof(double) * fv));
  MBC_TRY(res64.reserve(sizeof(double) * (fv + 3 * nv)));
  double *Fd = (double *)fbuf64.ptr;
  double *Wd = (double *)res64.ptr;
  double *Xd = Wd + fv;
  double *Rd = Xd + nv;
  double *Bd = Rd + nv;
  if (adjoint) permute_in<double>(*this, R, rhs, rhs_dt, Bd, st);
  else {
    load_rows<double>(*this, R, rhs, rhs_dt, Fd, st);
    launch_cols<double>(*this, R, Fd, Bd, nullptr, nullptr, nullptr, st);
  }
  if (X0) permute_in<double>(*this, R, X0, x_dt, Xd, st);
  else MBC_CK(cudaMemsetAsync(Xd, 0, sizeof(double) * nv, st));
  MBC_CKL();
  PcgWork<float> w;
  MBC_TRY(pcg_buffers<float>(*this, R, w));
  const Layout2D L = layout2d(n, R);
  // r64 = b - K^T K x64 (FP64), r = (float) r64
  auto true_residual_into_r = [&]() -> mbc_status {
    if (adjoint) {
      launch_rows<double>(*this, R, Xd, Wd, nullptr, st);
      launch_cols<double>(*this, R, Wd, Rd, nullptr, nullptr, nullptr, st);
      sub_kernel<double><<<cdiv(nv, 256), 256, 0, st>>>(nv, Bd, Rd, Rd);
      ++launches;
    } else {
      residual<double>(*this, R, Fd, Xd, Wd, Rd, st);
    }
    convert<double, float>((int64_t)nv, Rd, w.Rv, st);
    ++launches;
    MBC_CKL();
    return MBC_OK;
  };
  if (X0) MBC_TRY(true_residual_into_r());
  else {
    convert<double, float>((int64_t)nv, Bd, w.Rv, st);
    ++launches;
  }
  // thresholds relative to |b|^2 in FP64
  MBC_TRY(b2ref.reserve(sizeof(double) * R));
  MBC_TRY(col_norms2_dev<double>(*this, R, Bd, (double *)b2ref.ptr, st));
  std::function<mbc_status()> replace = [&]() -> mbc_status {
    MBC_TRY(true_residual_into_r());
    dot_partial_kernel<double><<<L.grid, L.block, L.smem, st>>>(n, R, Rd, Rd, w.part);
    reduce_kernel<<<1, 1024, 0, st>>>((int)L.grid.x, R, w.part, RED_REPLACE, w.sc, nullptr);
    launches += 2;
    MBC_CKL();
    return MBC_OK;
  };
  const double drop = std::min(std::max(o.inner_tol, 1e-6), 0.5);
  w.sc.drop2 = drop * drop;
  const int max_replace = o.max_refine > 0 ? std::max(o.max_refine, 1) : 0;
  MBC_TRY((run_pcg<float, float, double>(*this, R, w, Xd, (const float *)lval.ptr, o.max_iters, o.tol,
                                         o.precondition != 0, std::max(1, o.check_every), nullptr, st,
                                         (const double *)b2ref.ptr, &replace, max_replace)));
  // final true residual for every column (the status of columns that hit
  // max_iters is decided on it)
  MBC_TRY(replace());
  std::vector<int32_t> status, iters;
  std::vector<double> rel;
  MBC_TRY(collect<float>(*this, R, w, status, iters, rel, st));
  const int32_t n_repl = replacements;
  // columns the FP32 recursion could not finish (stagnant or out of
  // iterations) are polished by FP64 PCG warm-started from their FP64 x
  std::vector<int32_t> pol;
  for (int c = 0; c < R; ++c)
    if (status[c] == COL_STAGNANT || status[c] == COL_MAXIT) pol.push_back(c);
  const int32_t n_polished = (int32_t)pol.size();
  // With the INT8 FP64 operator a polish run stops on its recursive
  // residual, which can end just above tol once recomputed: such columns are
  // polished again from where they stand (at most twice more).
  const int passes = use_oz(*this) ? 3 : 1;
  for (int pass = 0; pass < passes && !pol.empty(); ++pass) {
    const int Rs = (int)pol.size();
    MBC_TRY(polish_idx.reserve(sizeof(int32_t) * (Rs + 2) + sizeof(double) * R));
    int32_t *d_idx = (int32_t *)polish_idx.ptr;
    MBC_CK(cudaMemcpyAsync(d_idx, pol.data(), sizeof(int32_t) * Rs, cudaMemcpyHostToDevice, st));
    PcgWork<double> w64;
    MBC_TRY(pcg_buffers<double>(*this, Rs, w64));
    const int64_t ns = (int64_t)n * Rs;
    gather_cols_kernel<double><<<cdiv(ns, 256), 256, 0, st>>>(n, R, Rs, d_idx, Xd, w64.X);
    gather_cols_kernel<double><<<cdiv(ns, 256), 256, 0, st>>>(n, R, Rs, d_idx, Rd, w64.Rv);
    std::vector<double> b2_all(R), b2_sel(Rs);
    MBC_CK(cudaMemcpyAsync(b2_all.data(), b2ref.ptr, sizeof(double) * R, cudaMemcpyDeviceToHost, st));
    MBC_CK(cudaStreamSynchronize(st));
    for (int k = 0; k < Rs; ++k) b2_sel[k] = b2_all[pol[k]];
    double *d_b2s = (double *)((int32_t *)polish_idx.ptr + ((Rs + 1) & ~1));
    MBC_CK(cudaMemcpyAsync(d_b2s, b2_sel.data(), sizeof(double) * Rs, cudaMemcpyHostToDevice, st));
    launches += 2;
    MBC_CKL();
    MBC_TRY((run_pcg<double, float, double>(*this, Rs, w64, w64.X, (const float *)lval.ptr,
                                            o.max_iters, o.tol, o.precondition != 0,
                                            std::max(1, o.check_every), nullptr, st, d_b2s, nullptr,
                                            0, o.compact != 0)));
    std::vector<int32_t> it64(Rs);
    MBC_CK(cudaMemcpyAsync(it64.data(), w64.sc.iters, sizeof(int32_t) * Rs, cudaMemcpyDeviceToHost, st));
    scatter_cols_kernel<double><<<cdiv(ns, 256), 256, 0, st>>>(n, R, Rs, d_idx, w64.X, Xd);
    ++launches;
    MBC_CKL();
    MBC_CK(cudaStreamSynchronize(st));
    for (int k = 0; k < Rs; ++k) iters[pol[k]] += it64[k];
    // every polished column is decided on its FP64 true residual
    MBC_TRY(true_residual_into_r());
    std::vector<double> nr, nb;
    MBC_TRY(col_norms2<double>(*this, R, Rd, nr, st));
    MBC_TRY(col_norms2<double>(*this, R, Bd, nb, st));
    std::vector<int32_t> again;
    for (int c : pol) {
      rel[c] = nb[c] < 1e-16 ? 0.0 : std::sqrt(nr[c] / nb[c]);
      status[c] = rel[c] <= o.tol ? COL_OK : COL_MAXIT;
      if (status[c] != COL_OK) again.push_back(c);
    }
    pol.swap(again);
  }
  permute_out<double>(*this, R, Xd, X, x_dt, st);
  MBC_CKL();
  for (int c = 0; c < R; ++c)
    if (status[c] == COL_STAGNANT) status[c] = COL_MAXIT;
  MBC_TRY(finish_stats(R, status, iters, rel, stats, iters_host));
  if (stats) {
    stats->n_polished = n_polished;
    stats->refinements = n_repl + 1;
    double m = 0;
    for (int c = 0; c < R; ++c) m = std::max(m, rel[c]);
    stats->true_relres_max = m;
    stats->relres_max = m;
  }
  MBC_CK(cudaStreamSynchronize(st));
  return MBC_OK;
}

template mbc_status Solver::solve_plain<float>(int, const void *, int32_t, void *, int32_t, const void *, bool,
                                               const mbc_solve_options &, mbc_solve_stats *, int32_t *, cudaStream_t);
template mbc_status Solver::solve_plain<double>(int, const void *, int32_t, void *, int32_t, const void *, bool,
                                                const mbc_solve_options &, mbc_solve_stats *, int32_t *, cudaStream_t);

mbc_status Solver::solve(int R, const void *rhs, int32_t rhs_dt, void *X, int32_t x_dt, const void *X0,
                         bool adjoint, const mbc_solve_options &o, mbc_solve_stats *stats,
                         int32_t *iters_host, cudaStream_t st)
{
  if (!factored) return fail(MBC_BAD_ARG, "solver is not factored (call mbc_solver_factor)");
  MBC_TRY(ensure_oz(st, R));
  oz_unprepared = false;
  const auto t0 = std::chrono::steady_clock::now();
  const int64_t launches0 = launches;
  profile = o.profile != 0;
  graph = o.graph != 0;
  prof_ms_all.clear();
  prof_is64.clear();
  prof_cols.clear();
  mbc_status rs;
  if (o.schedule == MBC_SCHED_PER_RHS && R > 1) {
    // one cold-started PCG per column, in order (mfs_torch_ops.cu:166-171)
    const size_t rows = adjoint ? (size_t)n : (size_t)nf;
    const size_t ein = rhs_dt == MBC_F64 ? 8 : 4, eout = x_dt == MBC_F64 ? 8 : 4;
    MBC_TRY(colbuf.reserve(rows * ein + (size_t)n * eout * 2));
    char *cin = (char *)colbuf.ptr;
    char *cx0 = cin + rows * ein;
    char *cout = cx0 + (size_t)n * eout;
    mbc_solve_stats agg{};
    agg.true_relres_max = -1;
    int worst = 0;
    rs = MBC_OK;
    for (int c = 0; c < R; ++c) {
      MBC_CK(cudaMemcpy2DAsync(cin, ein, (const char *)rhs + c * ein, ein * R, ein, rows,
                               cudaMemcpyDeviceToDevice, st));
      if (X0)
        MBC_CK(cudaMemcpy2DAsync(cx0, eout, (const char *)X0 + c * eout, eout * R, eout, n,
                                 cudaMemcpyDeviceToDevice, st));
      mbc_solve_stats s1{};
      int32_t it1 = 0;
      mbc_solve_options o1 = o;
      if (precision == MBC_F64 || o.fp64_recursion || o.max_refine <= 0)
        rs = (precision == MBC_F64 || o.fp64_recursion)
                 ? solve_plain<double>(1, cin, rhs_dt, cout, x_dt, X0 ? cx0 : nullptr, adjoint, o1, &s1, &it1, st)
                 : solve_plain<float>(1, cin, rhs_dt, cout, x_dt, X0 ? cx0 : nullptr, adjoint, o1, &s1, &it1, st);
      else
        rs = solve_mixed(1, cin, rhs_dt, cout, x_dt, X0 ? cx0 : nullptr, adjoint, o1, &s1, &it1, st);
      if (rs != MBC_OK) return rs;
      MBC_CK(cudaMemcpy2DAsync((char *)X + c * eout, eout * R, cout, eout, eout, n,
                               cudaMemcpyDeviceToDevice, st));
      if (iters_host) iters_host[c] = it1;
      agg.iters_max = std::max(agg.iters_max, s1.iters_max);
      agg.iters_total += s1.iters_total;
      agg.n_converged += s1.n_converged;
      agg.relres_max = std::max(agg.relres_max, s1.relres_max);
      agg.true_relres_max = std::max(agg.true_relres_max, s1.true_relres_max);
      agg.refinements = std::max(agg.refinements, s1.refinements);
      worst = std::max(worst, s1.status_per_worst);
    }
    agg.status_per_worst = worst;
    MBC_CK(cudaStreamSynchronize(st));
    if (stats) *stats = agg;
  } else if (precision == MBC_F64 || o.fp64_recursion) {
    // MBC_F32 with fp64_recursion: FP64 PCG preconditioned by the FP32 factor
    rs = solve_plain<double>(R, rhs, rhs_dt, X, x_dt, X0, adjoint, o, stats, iters_host, st);
  } else if (o.max_refine <= 0) {
    rs = solve_plain<float>(R, rhs, rhs_dt, X, x_dt, X0, adjoint, o, stats, iters_host, st);
  } else {
    rs = solve_mixed(R, rhs, rhs_dt, X, x_dt, X0, adjoint, o, stats, iters_host, st);
  }
  if (rs != MBC_OK) return rs;
  if (stats) {
    stats->t_solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    stats->kernel_launches = launches - launches0;
    stats->t_matvec_ms = 0;
    stats->n_matvec = 0;
    stats->t_matvec64_ms = 0;
    stats->n_matvec64 = 0;
    stats->matvec64_columns = 0;
    if (profile) {
      // a matvec pair whose kernels exited on the done flag takes a few
      // microseconds; count only pairs that did work (> 1% of the longest of
      // the same precision)
      float mx[2] = {0.f, 0.f};
      for (size_t i = 0; i < prof_ms_all.size(); ++i) mx[prof_is64[i]] = std::max(mx[prof_is64[i]], prof_ms_all[i]);
      for (size_t i = 0; i < prof_ms_all.size(); ++i) {
        const int p64 = prof_is64[i];
        if (prof_ms_all[i] > 0.01f * mx[p64]) {
          stats->t_matvec_ms += prof_ms_all[i];
          stats->n_matvec += 2;
          if (p64) {
            stats->t_matvec64_ms += prof_ms_all[i];
            stats->n_matvec64 += 2;
            stats->matvec64_columns += 2 * (int64_t)prof_cols[i];
          }
        }
      }
    }
  }
  MBC_TRY(check_device_error(st));
  if (stats && stats->status_per_worst == 2) return fail(MBC_BREAKDOWN, "PCG breakdown (p.Ap <= 0 or NaN)");
  if (stats && stats->status_per_worst == 1) return fail(MBC_NOT_CONVERGED, "PCG reached max_iters above tol");
  return MBC_OK;
}

}  // namespace mbc

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
using mbc::fail;


extern "C" mbc_status mbc_solver_create(const mbc_plan *plan, const mbc_operator *op, int32_t precision,
                                        mbc_stream stream, mbc_solver **out)
{
  if (!out) return fail(MBC_BAD_ARG, "out is NULL");
  *out = nullptr;
  if (!plan || !op) return fail(MBC_BAD_ARG, "NULL plan or operator");
  if (precision != MBC_F64 && precision != MBC_F32) return fail(MBC_BAD_ARG, "precision must be MBC_F64 or MBC_F32");
  if (op->n != plan->p.n || op->nf <= 0) return fail(MBC_BAD_ARG, "operator columns must equal the plan's points");
  if (op->kind == MBC_OP_DENSE) {
    if (!op->M || op->ldm < op->n) return fail(MBC_BAD_ARG, "dense operator needs M with ldm >= n");
  } else if (op->kind == MBC_OP_POINT_KERNEL) {
    if (!op->x || !op->nx || !op->y) return fail(MBC_BAD_ARG, "point kernel needs x, nx and y");
  } else if (op->kind == MBC_OP_MESH) {
    if (!op->V || !op->faces || !op->y || op->n_vert <= 0)
      return fail(MBC_BAD_ARG, "mesh operator needs V (n_vert > 0), faces and y");
  } else {
    return fail(MBC_BAD_ARG, "unknown operator kind");
  }
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) {
    cudaGetLastError();
    return fail(MBC_CUDA_ERROR, "no CUDA device");
  }
  std::unique_ptr<mbc_solver> sv(new (std::nothrow) mbc_solver());
  if (!sv) return fail(MBC_NO_MEMORY, "solver allocation failed");
  if (cudaMallocHost((void **)&sv->s.h_flag, sizeof(int32_t) * 4) != cudaSuccess) {
    cudaGetLastError();
    return fail(MBC_NO_MEMORY, "pinned flag allocation failed");
  }
  mbc_status s = sv->s.create(plan->p, *op, precision, (cudaStream_t)stream);
  if (s != MBC_OK) return s;
  *out = sv.release();
  return MBC_OK;
}

mbc::Solver::~Solver()
{
  if (h_flag) cudaFreeHost(h_flag);
  for (cudaEvent_t e : events) cudaEventDestroy(e);
}

mbc_status mbc::Solver::check_device_error(cudaStream_t st)
{
  if (oz_unprepared) {
    oz_unprepared = false;
    return fail(MBC_CUDA_ERROR, "an INT8 matvec found its buffers unsized and did not run");
  }
  int32_t e = 0;
  MBC_CK(cudaMemcpyAsync(&e, m_err.ptr, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  MBC_CK(cudaStreamSynchronize(st));
  if (e) {
    MBC_CK(cudaMemsetAsync(m_err.ptr, 0, sizeof(int32_t), st));
    if (e == 2) return fail(MBC_CUDA_ERROR, "tensor-core kernel: shared memory window not 1024-byte aligned");
    if (e == 3) return fail(MBC_BAD_ARG, "non-finite kernel value: a source coincides with a collocation point");
    if (e == 4)
      return fail(MBC_CUDA_ERROR, "tensor-core kernel: an index or size fell outside its buffer (the access was skipped)");
    return fail(MBC_TIMEOUT, "a bounded device wait expired in a tensor-core kernel");
  }
  return MBC_OK;
}

mbc_status mbc::Solver::ensure_events(int count)
{
  while ((int)events.size() < count) {
    cudaEvent_t e;
    MBC_CK(cudaEventCreate(&e));
    events.push_back(e);
  }
  return MBC_OK;
}

extern "C" mbc_status mbc_solver_destroy(mbc_solver *s)
{
  delete s;
  return MBC_OK;
}

extern "C" mbc_status mbc_solver_factor(mbc_solver *s, mbc_stream stream)
{
  if (!s) return fail(MBC_BAD_ARG, "NULL solver");
  return s->s.factor((cudaStream_t)stream);
}

extern "C" void mbc_factor_default_tiles(mbc_factor_tiles *t)
{
  if (!t) return;
  *t = mbc_factor_tiles{{32, 64, 128}, {64, 32, 32, 8}, 64};
}

static bool tiles_valid(const mbc_factor_tiles &t)
{
  if (t.max_ns[0] < 1 || t.max_ns[0] >= t.max_ns[1] || t.max_ns[1] >= t.max_ns[2] || t.max_ns[2] > 144) return false;
  for (int c = 0; c < 4; ++c)
    if (t.tile_rows[c] < 1 || t.tile_rows[c] > 256) return false;
  return t.tc_min_ns == 0 || (t.tc_min_ns >= mbc::ftc::kMinNs && t.tc_min_ns <= mbc::ftc::kMaxNs);
}

extern "C" mbc_status mbc_solver_set_factor_tiles(mbc_solver *s, const mbc_factor_tiles *t)
{
  if (!s || !t) return fail(MBC_BAD_ARG, "NULL solver or tiles");
  if (!tiles_valid(*t)) return fail(MBC_BAD_ARG, "factor tiles: need 1 <= max_ns[0] < max_ns[1] < max_ns[2] <= 144, "
                                                 "1 <= tile_rows <= 256 and tc_min_ns 0 or 32 .. 192");
  s->s.tiles = *t;
  return MBC_OK;
}

extern "C" mbc_status mbc_solver_get_factor_tiles(const mbc_solver *s, mbc_factor_tiles *t)
{
  if (!s || !t) return fail(MBC_BAD_ARG, "NULL solver or tiles");
  *t = s->s.tiles;
  return MBC_OK;
}

extern "C" mbc_status mbc_solver_tune_factor(mbc_solver *s, int32_t reps, mbc_factor_tiles *best_out,
                                             double *ms_best, mbc_stream stream)
{
  if (!s || reps < 1) return fail(MBC_BAD_ARG, "NULL solver or reps < 1");
  mbc::Solver &S = s->s;
  cudaStream_t st = (cudaStream_t)stream;
  cudaEvent_t e0, e1;
  MBC_CK(cudaEventCreate(&e0));
  MBC_CK(cudaEventCreate(&e1));
  struct Ev {
    cudaEvent_t a, b;
    ~Ev()
    {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  } ev{e0, e1};
  // the median of `reps` factor times of a candidate; +inf if it cannot run
  auto time_of = [&](const mbc_factor_tiles &t) -> double {
    if (!tiles_valid(t)) return INFINITY;
    S.tiles = t;
    std::vector<float> ms;
    for (int r = 0; r < reps; ++r) {
      cudaEventRecord(e0, st);
      if (S.factor(st) != MBC_OK) return INFINITY;
      cudaEventRecord(e1, st);
      if (cudaEventSynchronize(e1) != cudaSuccess) return INFINITY;
      float m = 0.f;
      cudaEventElapsedTime(&m, e0, e1);
      ms.push_back(m);
    }
    std::sort(ms.begin(), ms.end());
    return ms[ms.size() / 2];
  };
  mbc_factor_tiles best = S.tiles;
  double tbest = time_of(best);
  // class bounds, with the current panel rows
  const int b0s[3] = {24, 32, 48}, b1s[2] = {64, 96}, b2s[2] = {128, 144};
  for (int b0 : b0s)
    for (int b1 : b1s)
      for (int b2 : b2s) {
        mbc_factor_tiles t = best;
        t.max_ns[0] = b0;
        t.max_ns[1] = b1;
        t.max_ns[2] = b2;
        const double tm = time_of(t);
        if (tm < tbest) {
          tbest = tm;
          best = t;
        }
      }
  // the smallest set whose Gram runs on the tensor cores (FP32 factors)
  if (S.precision != MBC_F64) {
    const int mins[6] = {0, 32, 48, 64, 96, 128};
    for (int m : mins) {
      mbc_factor_tiles t = best;
      t.tc_min_ns = m;
      const double tm = time_of(t);
      if (tm < tbest) {
        tbest = tm;
        best = t;
      }
    }
  }
  // then the panel rows, one class at a time
  const int rows[5] = {8, 16, 32, 64, 128};
  for (int c = 0; c < 4; ++c)
    for (int r : rows) {
      mbc_factor_tiles t = best;
      t.tile_rows[c] = r;
      const double tm = time_of(t);
      if (tm < tbest) {
        tbest = tm;
        best = t;
      }
    }
  S.tiles = best;
  MBC_TRY(S.factor(st));
  MBC_CK(cudaStreamSynchronize(st));
  if (!std::isfinite(tbest)) return fail(MBC_CUDA_ERROR, "factor tuning: no candidate ran");
  if (best_out) *best_out = best;
  if (ms_best) *ms_best = tbest;
  return MBC_OK;
}

extern "C" mbc_status mbc_solver_set_wait_limit(mbc_solver *s, uint32_t polls)
{
  if (!s) return fail(MBC_BAD_ARG, "NULL solver");
  s->s.wait_limit = polls;
  return MBC_OK;
}

extern "C" mbc_status mbc_solver_get_tensor_grams(const mbc_solver *s, int32_t *count)
{
  if (!s || !count) return fail(MBC_BAD_ARG, "NULL solver or count");
  *count = s->s.gram_tc_count;
  return MBC_OK;
}

extern "C" mbc_status mbc_solver_get_factor(const mbc_solver *s, double *lval_host, double *theta_host)
{
  if (!s) return fail(MBC_BAD_ARG, "NULL solver");
  const mbc::Solver &S = s->s;
  if (!S.factored) return fail(MBC_BAD_ARG, "solver is not factored");
  const mbc::Plan &p = *S.plan;
  const size_t ln = (size_t)p.lptr.back(), tn = (size_t)p.th_ptr.back();
  auto fetch = [&](const void *src, size_t cnt, double *dst) -> mbc_status {
    if (S.precision == MBC_F64) {
      MBC_CK(cudaMemcpy(dst, src, cnt * sizeof(double), cudaMemcpyDeviceToHost));
    } else {
      std::vector<float> tmp(cnt);
      MBC_CK(cudaMemcpy(tmp.data(), src, cnt * sizeof(float), cudaMemcpyDeviceToHost));
      for (size_t k = 0; k < cnt; ++k) dst[k] = tmp[k];
    }
    return MBC_OK;
  };
  if (lval_host) MBC_TRY(fetch(S.lval.ptr, ln, lval_host));
  if (theta_host) MBC_TRY(fetch(S.theta.ptr, tn, theta_host));
  return MBC_OK;
}

extern "C" mbc_status mbc_solver_get_pivot_retries(const mbc_solver *s, int32_t *count)
{
  if (!s || !count) return fail(MBC_BAD_ARG, "NULL argument");
  *count = s->s.pivot_retries;
  return MBC_OK;
}

extern "C" mbc_status mbc_solver_set_matvec(mbc_solver *s, int32_t impl)
{
  if (!s) return fail(MBC_BAD_ARG, "NULL solver");
  if (impl < MBC_MATVEC_AUTO || impl > MBC_MATVEC_TENSOR) return fail(MBC_BAD_ARG, "unknown matvec implementation");
  s->s.matvec_impl = impl;
  return MBC_OK;
}

extern "C" void mbc_solve_default_options(mbc_solve_options *o)
{
  if (!o) return;
  o->max_iters = 1000;
  o->tol = 1e-8;
  o->schedule = MBC_SCHED_BATCHED;
  o->precondition = 1;
  o->max_refine = 64;
  o->inner_tol = 1e-2;
  o->check_every = 8;
  o->true_residual = 0;
  o->profile = 0;
  o->graph = 0;
  o->compact = 0;
  o->fp64_recursion = 0;
}

static mbc_status check_solve_args(mbc_solver *s, int32_t R, const void *in, int32_t in_dt, void *X,
                                   int32_t x_dt)
{
  if (!s) return fail(MBC_BAD_ARG, "NULL solver");
  if (R <= 0 || !in || !X) return fail(MBC_BAD_ARG, "need R > 0 and device arrays");
  if ((in_dt != MBC_F64 && in_dt != MBC_F32) || (x_dt != MBC_F64 && x_dt != MBC_F32))
    return fail(MBC_BAD_ARG, "dtype must be MBC_F64 or MBC_F32");
  return MBC_OK;
}

extern "C" mbc_status mbc_solve(mbc_solver *s, int32_t R, const void *F, int32_t f_dtype, void *X,
                                int32_t x_dtype, const void *X0, const mbc_solve_options *opt,
                                mbc_solve_stats *stats_host, int32_t *iters_host, mbc_stream stream)
{
  MBC_TRY(check_solve_args(s, R, F, f_dtype, X, x_dtype));
  mbc_solve_options o;
  mbc_solve_default_options(&o);
  if (opt) o = *opt;
  if (o.max_iters < 0 || !(o.tol >= 0)) return fail(MBC_BAD_ARG, "bad solve options");
  return s->s.solve(R, F, f_dtype, X, x_dtype, X0, false, o, stats_host, iters_host, (cudaStream_t)stream);
}

extern "C" mbc_status mbc_solve_adjoint(mbc_solver *s, int32_t R, const void *B, int32_t b_dtype, void *X,
                                        int32_t x_dtype, const mbc_solve_options *opt,
                                        mbc_solve_stats *stats_host, int32_t *iters_host, mbc_stream stream)
{
  MBC_TRY(check_solve_args(s, R, B, b_dtype, X, x_dtype));
  mbc_solve_options o;
  mbc_solve_default_options(&o);
  if (opt) o = *opt;
  if (o.max_iters < 0 || !(o.tol >= 0)) return fail(MBC_BAD_ARG, "bad solve options");
  return s->s.solve(R, B, b_dtype, X, x_dtype, nullptr, true, o, stats_host, iters_host, (cudaStream_t)stream);
}

extern "C" mbc_status mbc_apply_K(mbc_solver *s, int32_t R, const void *V, void *W, mbc_stream stream)
{
  if (!s || R <= 0 || !V || !W) return fail(MBC_BAD_ARG, "bad arguments");
  mbc::Solver &S = s->s;
  cudaStream_t st = (cudaStream_t)stream;
  if (S.precision == MBC_F64) {
    MBC_TRY(S.ensure_oz(st, R));
    MBC_TRY(S.tmp.reserve(sizeof(double) * (size_t)S.n * R));
    mbc::permute_in<double>(S, R, V, MBC_F64, (double *)S.tmp.ptr, st);
    mbc::launch_rows<double>(S, R, (const double *)S.tmp.ptr, (double *)W, nullptr, st);
  } else {
    MBC_TRY(S.tmp.reserve(sizeof(float) * (size_t)S.n * R));
    mbc::permute_in<float>(S, R, V, MBC_F32, (float *)S.tmp.ptr, st);
    mbc::launch_rows<float>(S, R, (const float *)S.tmp.ptr, (float *)W, nullptr, st);
  }
  MBC_CKL();
  return S.check_device_error(st);
}

extern "C" mbc_status mbc_apply_KT(mbc_solver *s, int32_t R, const void *W, void *T, mbc_stream stream)
{
  if (!s || R <= 0 || !W || !T) return fail(MBC_BAD_ARG, "bad arguments");
  mbc::Solver &S = s->s;
  cudaStream_t st = (cudaStream_t)stream;
  if (S.precision == MBC_F64) {
    MBC_TRY(S.ensure_oz(st, R));
    MBC_TRY(S.tmp.reserve(sizeof(double) * (size_t)S.n * R));
    mbc::launch_cols<double>(S, R, (const double *)W, (double *)S.tmp.ptr, nullptr, nullptr, nullptr, st);
    mbc::permute_out<double>(S, R, (const double *)S.tmp.ptr, T, MBC_F64, st);
  } else {
    MBC_TRY(S.tmp.reserve(sizeof(float) * (size_t)S.n * R));
    mbc::launch_cols<float>(S, R, (const float *)W, (float *)S.tmp.ptr, nullptr, nullptr, nullptr, st);
    mbc::permute_out<float>(S, R, (const float *)S.tmp.ptr, T, MBC_F32, st);
  }
  MBC_CKL();
  return S.check_device_error(st);
}

// Added-mass tensor and fluid forces from solved strengths (see mbc.h).
extern "C" mbc_status mbc_added_mass(mbc_solver *s, int32_t R, const void *X, int32_t x_dtype, const float *w,
                                     int32_t n_bodies, const int32_t *body_ptr, const double *centers,
                                     double rho_fluid, double *Mf, const double *accel, double *forces,
                                     mbc_stream stream)
{
  if (!s || R <= 0 || !X || !w || n_bodies <= 0 || !body_ptr || !centers || !Mf)
    return fail(MBC_BAD_ARG, "mbc_added_mass: NULL pointer or non-positive size");
  if (x_dtype != MBC_F32 && x_dtype != MBC_F64) return fail(MBC_BAD_ARG, "mbc_added_mass: bad x_dtype");
  if ((accel == nullptr) != (forces == nullptr))
    return fail(MBC_BAD_ARG, "mbc_added_mass: accel and forces go together");
  if (accel && R != 6 * n_bodies)
    return fail(MBC_BAD_ARG, "mbc_added_mass: forces need R == 6 * n_bodies (all rigid modes)");
  mbc::Solver &S = s->s;
  if (S.op.kind != MBC_OP_POINT_KERNEL)
    return fail(MBC_UNSUPPORTED, "mbc_added_mass: needs a point-kernel operator (source positions)");
  if (body_ptr[0] != 0) return fail(MBC_BAD_ARG, "mbc_added_mass: body_ptr[0] must be 0");
  for (int a = 0; a < n_bodies; ++a)
    if (body_ptr[a + 1] < body_ptr[a] || body_ptr[a + 1] > S.nf)
      return fail(MBC_BAD_ARG, "mbc_added_mass: body_ptr must ascend within [0, nf]");
  if ((R + 31) / 32 > 65535) return fail(MBC_BAD_ARG, "mbc_added_mass: R too large");
  cudaStream_t st = (cudaStream_t)stream;
  mbc::DevMem xp, phi, dmf, dptr, dcen;
  MBC_TRY(xp.reserve(sizeof(double) * (size_t)S.n * R));
  MBC_TRY(phi.reserve(sizeof(double) * (size_t)S.nf * R));
  MBC_TRY(dmf.reserve(sizeof(double) * (size_t)6 * n_bodies * R));
  MBC_TRY(dptr.reserve(sizeof(int32_t) * (size_t)(n_bodies + 1)));
  MBC_TRY(dcen.reserve(sizeof(double) * (size_t)3 * n_bodies));
  MBC_CK(cudaMemcpyAsync(dptr.ptr, body_ptr, sizeof(int32_t) * (n_bodies + 1), cudaMemcpyHostToDevice, st));
  MBC_CK(cudaMemcpyAsync(dcen.ptr, centers, sizeof(double) * 3 * n_bodies, cudaMemcpyHostToDevice, st));
  // phi = SL X in FP64 (strengths gathered into the plan order of the sources)
  mbc::permute_in<double>(S, R, X, x_dtype, (double *)xp.ptr, st);
  {
    constexpr int RC = 16, TI = 64;
    dim3 grid(mbc::cdiv(S.nf, TI), mbc::cdiv(R, RC));
    mbc::pk_rows_kernel<double, RC, TI, mbc::TJ_ROWS, mbc::SingleLayer64><<<grid, TI, 0, st>>>(
        S.x4(), S.n4(), S.nf, S.y4(), S.n, (const double *)xp.ptr, R, 1.0 / (4.0 * 3.14159265358979323846),
        (double *)phi.ptr, R, R, nullptr);
  }
  mbc::added_mass_kernel<<<dim3(n_bodies, mbc::cdiv(R, 32)), 256, 0, st>>>(
      S.x4(), S.n4(), w, (const int32_t *)dptr.ptr, (const double *)dcen.ptr, (const double *)phi.ptr, R,
      rho_fluid, (double *)dmf.ptr);
  MBC_CKL();
  MBC_CK(cudaMemcpyAsync(Mf, dmf.ptr, sizeof(double) * (size_t)6 * n_bodies * R, cudaMemcpyDeviceToHost, st));
  MBC_CK(cudaStreamSynchronize(st));
  if (accel) {
    // reactive force of the added mass: f = -Mf a
    for (int i = 0; i < 6 * n_bodies; ++i) {
      double f = 0.0;
      for (int j = 0; j < R; ++j) f += Mf[(size_t)i * R + j] * accel[j];
      forces[i] = -f;
    }
  }
  return S.check_device_error(st);
}
