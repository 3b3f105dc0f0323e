// Supernodal KL factor, one CTA per supernode s:
//   1. Theta_s = K(:, I_s)^T K(:, I_s) over all nf collocation rows, written
//      in reversed order, column-major (kl_chol.cu:166-223); the K panels are
//      generated tile by tile in shared memory and never stored;
//   2. Theta_rev = U^T U in place, U in the upper triangle (kl_chol.cu:16-36),
//      right-looking so each step is a parallel rank-1 update;
//   3. every column c of s: L(:,c) = reverse(U_nb^-1 e_nb) on the leading
//      nb x nb block, nb = |column c| (kl_chol.cu:38-53, :362-387), one warp
//      per column.
// Theta_s stays in shared memory when it fits; larger supernodes work in
// their slice of the global Theta array instead.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "matvec.cuh"
#include "matvec_mesh.cuh"

namespace mbc {

struct FactorArgs {
  const int32_t *list;  // supernodes handled by this launch
  int32_t count;
  const int32_t *sup_ptr, *sup_ind, *set_ptr, *set_ind, *lptr;
  const int64_t *th_ptr;
  // operator
  int32_t kind;  // 0 dense, 1 point kernel, 2 mesh (solid angles)
  const float4 *xr, *nr, *ys;  // point kernel (ys in the new order); mesh: face vertices 1, 2
  const float4 *zr;            // mesh: face vertex 3
  const float *M;
  int64_t ldm;
  const int32_t *Pinv;  // dense: column of M for each new index
  int32_t nf;
  double coef;
  double shift;      // relative diagonal shift (retries only)
  // A pivot that keeps less than pivot_tol of its original diagonal entry
  // has cancelled most of its digits: the supernode is flagged for the FP64
  // retry (FP32 launches); 0 flags only non-positive pivots.
  double pivot_tol;
  // 1: Theta_s of every supernode of the launch is already in the global
  // Theta array (gram_tc_kernel, FP32 launches): step 1 only loads it
  int32_t gram_ready;
  int32_t smem_cap;  // largest n_s kept in shared memory
  int32_t tile_rows; // panel rows per tile
  int32_t *bad_list, *bad_count;
  // supernodes above smem_cap keep their warp buffers in global scratch:
  // (NT/32) * gscratch_stride elements per CTA
  void *gscratch;
  int64_t gscratch_stride;
};

__device__ __forceinline__ void tri_decode(int e, int &p, int &q)
{
  // e = q (q + 1) / 2 + p with 0 <= p <= q
  int qq = (int)((sqrtf(8.0f * (float)e + 1.0f) - 1.0f) * 0.5f);
  while ((qq + 1) * (qq + 2) / 2 <= e) ++qq;
  while (qq * (qq + 1) / 2 > e) --qq;
  q = qq;
  p = e - qq * (qq + 1) / 2;
}

template <typename T, typename LT, int NT, int EPT>
__global__ void __launch_bounds__(NT) factor_kernel(FactorArgs a, T *__restrict__ theta,
                                                     LT *__restrict__ lval)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int s = a.list[blockIdx.x];
  const int sb = a.set_ptr[s];
  const int ns = a.set_ptr[s + 1] - sb;
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int TR = a.tile_rows;

  // shared layout: [src coords or M columns][panel TR x ns][warp buffers][Theta?]
  unsigned char *sp = smem_raw;
  float4 *s_src = reinterpret_cast<float4 *>(sp);
  int32_t *s_col = reinterpret_cast<int32_t *>(sp);
  sp += ((size_t)ns * sizeof(float4) + 15) & ~(size_t)15;
  T *panel = reinterpret_cast<T *>(sp);
  sp += ((size_t)TR * ns * sizeof(T) + 15) & ~(size_t)15;
  const bool in_smem = ns <= a.smem_cap;
  T *wbuf;
  if (in_smem) {
    wbuf = reinterpret_cast<T *>(sp);
    sp += ((size_t)(NT / 32) * ns * sizeof(T) + 15) & ~(size_t)15;
  } else {
    wbuf = reinterpret_cast<T *>(a.gscratch) + (size_t)blockIdx.x * (NT / 32) * a.gscratch_stride;
  }
  T *A = in_smem ? reinterpret_cast<T *>(sp) : theta + a.th_ptr[s];

  for (int p = tid; p < ns; p += NT) {
    const int c = a.set_ind[sb + p];
    if (a.kind != 0) s_src[p] = a.ys[c];
    else s_col[p] = a.Pinv[c];
  }
  const int ne = ns * (ns + 1) / 2;
  const int groups = ne >= NT ? 1 : NT / ne;
  const int g = ne >= NT ? 0 : tid / ne;
  const bool in_group = g < groups;
  const T coef = (T)a.coef;
  __syncthreads();

  // 1. Gram assembly, entry chunks of NT*EPT upper-triangle entries (or,
  // with gram_ready, the tensor-core Gram from the global slice)
  if (a.gram_ready && in_smem) {
    const T *src = theta + a.th_ptr[s];
    for (int e = tid; e < ns * ns; e += NT) A[e] = src[e];
  }
  for (int e0 = 0; e0 < (a.gram_ready ? 0 : ne); e0 += NT * EPT) {
    int pe[EPT], qe[EPT];
    T acc[EPT];
#pragma unroll
    for (int k = 0; k < EPT; ++k) {
      const int e = e0 + (groups > 1 ? tid % ne : tid + k * NT);
      acc[k] = T(0);
      pe[k] = -1;
      qe[k] = 0;
      if (in_group && e < ne && (groups == 1 || k == 0)) tri_decode(e, pe[k], qe[k]);
    }
    for (int i0 = 0; i0 < a.nf; i0 += TR) {
      const int im = min(TR, a.nf - i0);
      __syncthreads();
      for (int t = tid; t < im * ns; t += NT) {
        const int rr = t / ns, p = t - rr * ns;
        const int i = i0 + rr;
        T kv;
        if (a.kind == 1) kv = coef * PointKernel<T>::eval(a.xr[i], a.nr[i], s_src[p]);
        else if (a.kind == 2) kv = coef * SolidAngle<T>::eval(a.xr[i], a.nr[i], a.zr[i], s_src[p]);
        else kv = (T)__ldg(a.M + (size_t)i * a.ldm + s_col[p]);
        panel[t] = kv;
      }
      __syncthreads();
      if (in_group) {
#pragma unroll
        for (int k = 0; k < EPT; ++k) {
          if (pe[k] < 0) continue;
          const T *cp = panel + pe[k], *cq = panel + qe[k];
          T sacc = acc[k];
          for (int rr = g; rr < im; rr += groups) sacc = fma(cp[rr * ns], cq[rr * ns], sacc);
          acc[k] = sacc;
        }
      }
    }
    // deterministic reduction over row groups into A (reversed, symmetric)
    for (int gg = 0; gg < groups; ++gg) {
      __syncthreads();
      if (in_group && g == gg) {
#pragma unroll
        for (int k = 0; k < EPT; ++k) {
          if (pe[k] < 0) continue;
          const int rp = ns - 1 - pe[k], rq = ns - 1 - qe[k];
          T v = acc[k];
          if (gg > 0) v += A[rp + (size_t)rq * ns];
          A[rp + (size_t)rq * ns] = v;
          A[rq + (size_t)rp * ns] = v;
        }
      }
    }
  }
  __syncthreads();

  // optional diagonal shift (retry path): shift * max diagonal
  __shared__ T s_scal[2];
  __shared__ int s_bad;
  if (tid == 0) {
    s_bad = 0;
    T dmax = T(0);
    for (int k = 0; k < ns; ++k) dmax = max(dmax, A[k + (size_t)k * ns]);
    s_scal[1] = (T)a.shift * dmax;
  }
  __syncthreads();
  if (a.shift > 0)
    for (int k = tid; k < ns; k += NT) A[k + (size_t)k * ns] += s_scal[1];
  // keep the diagonal for the cancellation test (wbuf is free until step 3)
  for (int k = tid; k < ns; k += NT) wbuf[k] = A[k + (size_t)k * ns];

  // 2. right-looking U^T U on the upper triangle
  for (int k = 0; k < ns; ++k) {
    __syncthreads();
    if (tid == 0) {
      const T d = A[k + (size_t)k * ns];
      if (!(d > T(0)) || d < (T)a.pivot_tol * wbuf[k]) s_bad = 1;
      const T u = sqrt(d > T(0) ? d : T(1));
      A[k + (size_t)k * ns] = u;
      s_scal[0] = T(1) / u;
    }
    __syncthreads();
    const T inv = s_scal[0];
    for (int j = k + 1 + tid; j < ns; j += NT) A[k + (size_t)j * ns] *= inv;
    __syncthreads();
    const int m = ns - k - 1;
    const int nt = m * (m + 1) / 2;
    for (int e = tid; e < nt; e += NT) {
      int pi, qj;
      tri_decode(e, pi, qj);
      const int i = k + 1 + pi, j = k + 1 + qj;
      A[i + (size_t)j * ns] -= A[k + (size_t)i * ns] * A[k + (size_t)j * ns];
    }
  }
  __syncthreads();
  if (s_bad) {
    if (tid == 0) {
      const int slot = atomicAdd(a.bad_count, 1);
      a.bad_list[slot] = s;
    }
    return;
  }

  // 3. KL columns, one warp per column
  T *buf = wbuf + (size_t)warp * (in_smem ? ns : a.gscratch_stride);
  const int c0 = a.sup_ptr[s], c1 = a.sup_ptr[s + 1];
  for (int cc = c0 + warp; cc < c1; cc += NT / 32) {
    const int c = a.sup_ind[cc];
    const int lb = a.lptr[c], nb = a.lptr[c + 1] - lb;
    for (int i = lane; i < nb; i += 32) buf[i] = (i == nb - 1) ? T(1) : T(0);
    for (int m = nb - 1; m >= 0; --m) {
      __syncwarp();
      const T ym = buf[m] / A[m + (size_t)m * ns];
      __syncwarp();
      if (lane == 0) buf[m] = ym;
      for (int i = lane; i < m; i += 32) buf[i] -= A[i + (size_t)m * ns] * ym;
    }
    __syncwarp();
    for (int k = lane; k < nb; k += 32) lval[lb + k] = (LT)buf[nb - 1 - k];
  }
  // keep the factored Theta (U above, Theta below) for parity checks
  if (in_smem && theta) {
    T *dst = theta + a.th_ptr[s];
    for (int e = tid; e < ns * ns; e += NT) dst[e] = A[e];
  }
}

}  // namespace mbc
