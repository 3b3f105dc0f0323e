// Device solver object behind mbc_solver.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "mbc_internal.h"

namespace mbc {

// Owned device allocation that only grows.
struct DevMem {
  void *ptr = nullptr;
  size_t bytes = 0;
  DevMem() = default;
  DevMem(const DevMem &) = delete;
  DevMem &operator=(const DevMem &) = delete;
  ~DevMem();
  mbc_status reserve(size_t b);
  void release();
};

struct Solver {
  const Plan *plan = nullptr;
  mbc_operator op{};
  int32_t precision = MBC_F64;
  int32_t n = 0, nf = 0;
  bool factored = false;
  int32_t pivot_retries = 0;
  int32_t *h_flag = nullptr;  // pinned
  mutable int64_t launches = 0;  // kernels launched by this solver
  int32_t replacements = 0;   // residual replacements in the last PCG run
  bool profile = false;
  bool graph = false;  // replay PCG iteration blocks as CUDA graphs
  int32_t matvec_impl = MBC_MATVEC_AUTO;
  int32_t fp64_matvec = MBC_FP64_MATVEC_SIMT;
  mbc_factor_tiles tiles{{32, 64, 128}, {64, 32, 32, 8}, 64};  // factor class bounds, panel rows, tensor Gram
  bool oz_ready = false;  // INT8 digit planes of G built for the current geometry
  mutable bool oz_unprepared = false;  // an INT8 launch found its buffers unsized (not run)
  bool oz_slab = false;   // planes rebuilt per matvec, slab by slab (they do not all fit)
  int oz_slab_tiles[2] = {0, 0};  // row tiles per slab, per direction
  std::vector<cudaEvent_t> events;
  std::vector<float> prof_ms_all;
  std::vector<int> prof_is64;  // 1: the pair ran in FP64
  std::vector<int> prof_cols;  // columns the pair carried

  // plan on the device
  DevMem m_P, m_Pinv, m_sup_ptr, m_sup_ind, m_set_ptr, m_set_ind, m_lptr, m_lind, m_rptr, m_rcol,
      m_rmap, m_th_ptr;
  DevMem class_list[4];
  DevMem class_list_tc[4], gram_list;  // FP32 factor: supernodes whose Gram ran on the tensor cores
  int32_t gram_tc_count = 0;           // supernodes of the last factor with the tensor-core Gram
  // operator: rows (original order) and sources (new order) as float4
  DevMem m_x4, m_n4, m_y4;
  DevMem m_z4;  // mesh operator: third vertex of every face (x4, n4 hold the first two)
  DevMem m_err;           // set by a tensor-core kernel (1: a bounded wait expired)
  uint32_t wait_limit = 0;  // polls before a tensor-core kernel's partner wait gives up (0: the default)
  mutable DevMem m_bimg;  // packed TF32 hi/lo image of the tensor-core B operand
  // FP64-accurate INT8 matvec: digit planes and exponents of G per direction
  // (0: rows, 1: columns), and the per-launch digit image of the vector block
  DevMem m_oz_a[2], m_oz_aexp[2];
  mutable DevMem m_oz_b, m_oz_bexp;
  // the reduction axes of the INT8 planes walk the points in Morton order:
  // m_oz_q[0][k] = plan position of the k-th source (K direction), m_oz_q[1][k]
  // = the k-th collocation row (K^T direction); the coordinates in that
  // order; the vector block gathered into it for each matvec
  DevMem m_oz_q[2], m_oz_ys, m_oz_xr, m_oz_nr;
  mutable DevMem m_oz_v;
  DevMem m_oz_chk;  // the self-check's vectors
  // factor
  DevMem theta, theta64, lval, bad, fscratch;
  // PCG workspaces
  DevMem work32, work64, part, scal, fbuf32, fbuf64, res64, mask, colbuf, tmp, b2ref, nrm, polish_idx;
  DevMem blk;  // block PCG: compact column blocks, search blocks, small matrices

  ~Solver();

  const int32_t *dP() const { return (const int32_t *)m_P.ptr; }
  const int32_t *d_Pinv() const { return (const int32_t *)m_Pinv.ptr; }
  const int32_t *d_sup_ptr() const { return (const int32_t *)m_sup_ptr.ptr; }
  const int32_t *d_sup_ind() const { return (const int32_t *)m_sup_ind.ptr; }
  const int32_t *d_set_ptr() const { return (const int32_t *)m_set_ptr.ptr; }
  const int32_t *d_set_ind() const { return (const int32_t *)m_set_ind.ptr; }
  const int32_t *d_lptr() const { return (const int32_t *)m_lptr.ptr; }
  const int32_t *d_lind() const { return (const int32_t *)m_lind.ptr; }
  const int32_t *d_rptr() const { return (const int32_t *)m_rptr.ptr; }
  const int32_t *d_rcol() const { return (const int32_t *)m_rcol.ptr; }
  const int32_t *d_rmap() const { return (const int32_t *)m_rmap.ptr; }
  const int64_t *d_th_ptr() const { return (const int64_t *)m_th_ptr.ptr; }
  const float4 *x4() const { return (const float4 *)m_x4.ptr; }
  const float4 *n4() const { return (const float4 *)m_n4.ptr; }
  const float4 *y4() const { return (const float4 *)m_y4.ptr; }
  const float4 *z4() const { return (const float4 *)m_z4.ptr; }

  mbc_status create(const Plan &pl, const mbc_operator &o, int32_t prec, cudaStream_t st);
  mbc_status ensure_events(int count);
  mbc_status check_device_error(cudaStream_t st);
  // INT8 FP64 matvec selected: build the digit planes if missing and size the
  // vector image for R columns (no-op otherwise)
  mbc_status ensure_oz(cudaStream_t st, int R);
  // one column through K and K^T with the INT8 and with the FP64 kernels
  mbc_status oz_selfcheck(cudaStream_t st);
  mbc_status factor(cudaStream_t st);
  mbc_status solve(int R, const void *rhs, int32_t rhs_dt, void *X, int32_t x_dt, const void *X0,
                   bool adjoint, const mbc_solve_options &o, mbc_solve_stats *stats,
                   int32_t *iters_host, cudaStream_t st);
  template <typename T>
  mbc_status solve_plain(int R, const void *rhs, int32_t rhs_dt, void *X, int32_t x_dt,
                         const void *X0, bool adjoint, const mbc_solve_options &o,
                         mbc_solve_stats *stats, int32_t *iters_host, cudaStream_t st);
  mbc_status solve_mixed(int R, const void *rhs, int32_t rhs_dt, void *X, int32_t x_dt,
                         const void *X0, bool adjoint, const mbc_solve_options &o,
                         mbc_solve_stats *stats, int32_t *iters_host, cudaStream_t st);
  mbc_status true_residual(int R, const void *F, int32_t f_dt, const void *X, int32_t x_dt,
                           mbc_solve_stats *stats, cudaStream_t st);
};

template <typename T>
void launch_rows(const Solver &S, int R, const T *v, T *w, const int32_t *done, cudaStream_t st);
template <typename T>
int launch_cols(const Solver &S, int R, const T *w, T *t, const T *pdot, double *part,
                const int32_t *done, cudaStream_t st);

}  // namespace mbc

// The C handle behind mbc_solver.
struct mbc_solver {
  mbc::Solver s;
};
