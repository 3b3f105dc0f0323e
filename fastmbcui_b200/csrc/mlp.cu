// mlp.cu -- the warm-start network: a small MLP trained and evaluated on the
// GPU by the kernels below (no library GEMM).
//
// Layers: n_in -> hidden x n_hidden_layers (tanh) -> n_out (linear).  Weights
// are kept as an FP32 master copy for training and as BF16 for the forward
// pass; every product accumulates in FP32.  Training minimises the mean
// squared error 0.5 * mean((y - t)^2) with Adam.  All reductions run in a
// fixed order, so a training step is deterministic.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "mbc_internal.h"
#include "solver.h"

namespace {

using mbc::DevMem;
using mbc::fail;

#define MLP_CK(call)                                                                   \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess) return fail(MBC_CUDA_ERROR, std::string(#call ": ") + cudaGetErrorString(e_)); \
  } while (0)
#define MLP_TRY(expr)            \
  do {                           \
    mbc_status s_ = (expr);      \
    if (s_ != MBC_OK) return s_; \
  } while (0)

inline unsigned cdiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

template <typename T>
__device__ __forceinline__ float ld(const T *p);
template <>
__device__ __forceinline__ float ld<float>(const float *p) { return *p; }
template <>
__device__ __forceinline__ float ld<__nv_bfloat16>(const __nv_bfloat16 *p) { return __bfloat162float(*p); }

enum Epi { EPI_NONE = 0, EPI_BIAS = 1, EPI_BIAS_TANH = 2, EPI_TANH_GRAD = 3 };

// C[m, n] = sum_k A[m*sam + k*sak] * B[k*sbk + n*sbn], FP32 accumulate, with
// an epilogue: + bias[n]; tanh; or * (1 - Y[m, n]^2) (the tanh derivative
// through the stored activation Y).  64 x 64 tile per block, 256 threads,
// 4 x 4 outputs per thread, k-tiles of 16 staged in shared memory.
template <typename TB>
__global__ void __launch_bounds__(256) gemm_kernel(int M, int N, int K, const float *__restrict__ A, int64_t sam,
                                                   int64_t sak, const TB *__restrict__ B, int64_t sbk, int64_t sbn,
                                                   float *__restrict__ C, int ldc, int epi,
                                                   const float *__restrict__ bias, const float *__restrict__ Y)
{
  __shared__ float sA[16][64 + 1];
  __shared__ float sB[16][64 + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += 16) {
    for (int t = threadIdx.x; t < 16 * 64; t += 256) {
      const int kk = t & 15, mm = t >> 4;
      const int gm = m0 + mm, gk = k0 + kk;
      sA[kk][mm] = (gm < M && gk < K) ? A[gm * sam + gk * sak] : 0.f;
      const int nn = t >> 4;
      const int gn = n0 + nn;
      sB[kk][nn] = (gn < N && gk < K) ? ld<TB>(B + gk * sbk + gn * sbn) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = sA[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = sB[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int gm = m0 + ty * 4 + i;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gn = n0 + tx * 4 + j;
      if (gn >= N) continue;
      float v = acc[i][j];
      if (epi == EPI_BIAS || epi == EPI_BIAS_TANH) v += bias[gn];
      if (epi == EPI_BIAS_TANH) v = tanhf(v);
      if (epi == EPI_TANH_GRAD) {
        const float y = Y[(int64_t)gm * ldc + gn];
        v *= 1.f - y * y;
      }
      C[(int64_t)gm * ldc + gn] = v;
    }
  }
}

// column sums of G (B x N) in a fixed order: one thread per column
__global__ void colsum_kernel(int Bn, int N, const float *__restrict__ G, float *__restrict__ out)
{
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.f;
  for (int b = 0; b < Bn; ++b) s += G[(int64_t)b * N + n];
  out[n] = s;
}

// G = (Y - T) / (B * N) and the per-block partial sums of 0.5 (Y - T)^2
__global__ void mse_grad_kernel(int64_t cnt, float scale, const float *__restrict__ Y, const float *__restrict__ T,
                                float *__restrict__ G, double *__restrict__ part)
{
  __shared__ double red[256];
  const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
  double e = 0.0;
  if (i < cnt) {
    const float d = Y[i] - T[i];
    G[i] = d * scale;
    e = 0.5 * (double)d * (double)d;
  }
  red[threadIdx.x] = e;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void sum_parts_kernel(int nb, const double *__restrict__ part, double scale, double *__restrict__ out)
{
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < nb; ++i) s += part[i];
    *out = s * scale;
  }
}

// Adam on the FP32 master parameters, then the BF16 copy of the weights
__global__ void adam_kernel(int64_t cnt, float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, __nv_bfloat16 *__restrict__ wb, float lr, float b1, float b2,
                            float eps, float c1, float c2)
{
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cnt) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  wb[i] = __float2bfloat16_rn(wi);
}

__global__ void to_bf16_kernel(int64_t cnt, const float *__restrict__ w, __nv_bfloat16 *__restrict__ wb)
{
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < cnt) wb[i] = __float2bfloat16_rn(w[i]);
}

}  // namespace

struct mbc_mlp {
  std::vector<int> dims;          // n_in, hidden..., n_out
  std::vector<int64_t> woff, boff;  // offsets of W_l (dims[l+1] x dims[l]) and b_l in the parameter vector
  int64_t n_params = 0;
  DevMem w, g, m, v, wb;          // FP32 master, gradients, Adam moments; BF16 weights
  DevMem acts, grads, part, loss; // activations per layer (B x dims[l]), pre-activation gradients
  int64_t steps = 0;
  int cap_batch = 0;
  int layers() const { return (int)dims.size() - 1; }
  int64_t act_off(int l, int B) const
  {
    int64_t o = 0;
    for (int i = 0; i < l; ++i) o += (int64_t)B * dims[i];
    return o;
  }
  mbc_status reserve_batch(int B)
  {
    if (B <= cap_batch) return MBC_OK;
    int64_t tot = 0, mx = 0;
    for (int d : dims) {
      tot += (int64_t)B * d;
      mx = std::max<int64_t>(mx, (int64_t)B * d);
    }
    MLP_TRY(acts.reserve(sizeof(float) * tot));
    MLP_TRY(grads.reserve(sizeof(float) * 2 * mx));
    MLP_TRY(part.reserve(sizeof(double) * (size_t)cdiv(mx, 256)));
    cap_batch = B;
    return MBC_OK;
  }
};

namespace {

template <typename TB>
void gemm(cudaStream_t st, int M, int N, int K, const float *A, int64_t sam, int64_t sak, const TB *B, int64_t sbk,
          int64_t sbn, float *C, int ldc, int epi, const float *bias, const float *Y)
{
  dim3 grid(cdiv(N, 64), cdiv(M, 64));
  gemm_kernel<TB><<<grid, 256, 0, st>>>(M, N, K, A, sam, sak, B, sbk, sbn, C, ldc, epi, bias, Y);
}

// forward through every layer; activations of layer l at acts + act_off(l)
void forward(mbc_mlp &net, int B, const float *X, float *Yout, cudaStream_t st)
{
  float *acts = (float *)net.acts.ptr;
  const __nv_bfloat16 *wb = (const __nv_bfloat16 *)net.wb.ptr;
  const float *w = (const float *)net.w.ptr;
  const float *in = X;
  for (int l = 0; l < net.layers(); ++l) {
    const int K = net.dims[l], N = net.dims[l + 1];
    const bool last = l == net.layers() - 1;
    float *out = last && Yout ? Yout : acts + net.act_off(l + 1, B);
    // out[b, n] = sum_k in[b, k] W[n, k] + bias[n]
    gemm<__nv_bfloat16>(st, B, N, K, in, K, 1, wb + net.woff[l], 1, K, out, N, last ? EPI_BIAS : EPI_BIAS_TANH,
                        w + net.boff[l], nullptr);
    in = out;
  }
}

}  // namespace

extern "C" mbc_status mbc_mlp_create(int32_t n_in, int32_t hidden, int32_t n_hidden_layers, int32_t n_out,
                                     uint64_t seed, mbc_mlp **out)
{
  if (!out || n_in <= 0 || hidden <= 0 || n_hidden_layers <= 0 || n_out <= 0)
    return fail(MBC_BAD_ARG, "mbc_mlp_create: bad sizes");
  *out = nullptr;
  auto net = new mbc_mlp();
  net->dims.push_back(n_in);
  for (int i = 0; i < n_hidden_layers; ++i) net->dims.push_back(hidden);
  net->dims.push_back(n_out);
  int64_t off = 0;
  for (int l = 0; l < net->layers(); ++l) {
    net->woff.push_back(off);
    off += (int64_t)net->dims[l + 1] * net->dims[l];
    net->boff.push_back(off);
    off += net->dims[l + 1];
  }
  net->n_params = off;
  // Glorot-uniform weights, zero biases, from the seed
  std::vector<float> h(off, 0.f);
  std::mt19937_64 rng(seed);
  for (int l = 0; l < net->layers(); ++l) {
    const double a = std::sqrt(6.0 / (net->dims[l] + net->dims[l + 1]));
    std::uniform_real_distribution<double> U(-a, a);
    for (int64_t i = 0; i < (int64_t)net->dims[l + 1] * net->dims[l]; ++i) h[net->woff[l] + i] = (float)U(rng);
  }
  mbc_status s = MBC_OK;
  if ((s = net->w.reserve(4 * off)) || (s = net->g.reserve(4 * off)) || (s = net->m.reserve(4 * off)) ||
      (s = net->v.reserve(4 * off)) || (s = net->wb.reserve(2 * off)) || (s = net->loss.reserve(8))) {
    delete net;
    return s;
  }
  cudaError_t e = cudaMemcpy(net->w.ptr, h.data(), 4 * off, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(net->m.ptr, 0, 4 * off);
  if (e == cudaSuccess) e = cudaMemset(net->v.ptr, 0, 4 * off);
  if (e == cudaSuccess) {
    to_bf16_kernel<<<cdiv(off, 256), 256>>>(off, (const float *)net->w.ptr, (__nv_bfloat16 *)net->wb.ptr);
    e = cudaDeviceSynchronize();
  }
  if (e != cudaSuccess) {
    delete net;
    return fail(MBC_CUDA_ERROR, std::string("mbc_mlp_create: ") + cudaGetErrorString(e));
  }
  *out = net;
  return MBC_OK;
}

extern "C" mbc_status mbc_mlp_destroy(mbc_mlp *net)
{
  delete net;
  return MBC_OK;
}

extern "C" mbc_status mbc_mlp_num_params(const mbc_mlp *net, int64_t *count)
{
  if (!net || !count) return fail(MBC_BAD_ARG, "mbc_mlp_num_params: NULL");
  *count = net->n_params;
  return MBC_OK;
}

// params_host: FP32, per layer W_l (row-major dims[l+1] x dims[l]) then b_l
extern "C" mbc_status mbc_mlp_get_params(const mbc_mlp *net, float *params_host)
{
  if (!net || !params_host) return fail(MBC_BAD_ARG, "mbc_mlp_get_params: NULL");
  MLP_CK(cudaMemcpy(params_host, net->w.ptr, 4 * net->n_params, cudaMemcpyDeviceToHost));
  return MBC_OK;
}

extern "C" mbc_status mbc_mlp_set_params(mbc_mlp *net, const float *params_host)
{
  if (!net || !params_host) return fail(MBC_BAD_ARG, "mbc_mlp_set_params: NULL");
  MLP_CK(cudaMemcpy(net->w.ptr, params_host, 4 * net->n_params, cudaMemcpyHostToDevice));
  to_bf16_kernel<<<cdiv(net->n_params, 256), 256>>>(net->n_params, (const float *)net->w.ptr,
                                                     (__nv_bfloat16 *)net->wb.ptr);
  MLP_CK(cudaGetLastError());
  MLP_CK(cudaDeviceSynchronize());
  return MBC_OK;
}

extern "C" mbc_status mbc_mlp_forward(mbc_mlp *net, int32_t batch, const float *X, float *Y, mbc_stream stream)
{
  if (!net || batch <= 0 || !X || !Y) return fail(MBC_BAD_ARG, "mbc_mlp_forward: bad arguments");
  MLP_TRY(net->reserve_batch(batch));
  forward(*net, batch, X, Y, (cudaStream_t)stream);
  MLP_CK(cudaGetLastError());
  return MBC_OK;
}

// One training step on (X, T): forward, MSE loss, backward into the gradient
// buffer, and (lr > 0) an Adam update.  loss_host (optional) receives the
// loss of this batch before the update; grads_host (optional) the gradient.
extern "C" mbc_status mbc_mlp_train_step(mbc_mlp *net, int32_t batch, const float *X, const float *T, float lr,
                                         double *loss_host, float *grads_host, mbc_stream stream)
{
  if (!net || batch <= 0 || !X || !T) return fail(MBC_BAD_ARG, "mbc_mlp_train_step: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  const int B = batch, L = net->layers();
  MLP_TRY(net->reserve_batch(B));
  float *acts = (float *)net->acts.ptr;
  float *g = (float *)net->g.ptr;
  const float *w = (const float *)net->w.ptr;
  const __nv_bfloat16 *wb = (const __nv_bfloat16 *)net->wb.ptr;
  // forward: layer l's input is X (l = 0) or acts[l]; the output layer goes to acts[L]
  const float *in = X;
  for (int l = 0; l < L; ++l) {
    const int K = net->dims[l], N = net->dims[l + 1];
    float *out = acts + net->act_off(l + 1, B);
    gemm<__nv_bfloat16>(st, B, N, K, in, K, 1, wb + net->woff[l], 1, K, out, N,
                        l == L - 1 ? EPI_BIAS : EPI_BIAS_TANH, w + net->boff[l], nullptr);
    in = out;
  }
  const int no = net->dims[L];
  const int64_t cnt = (int64_t)B * no;
  int64_t mx = 0;
  for (int d : net->dims) mx = std::max<int64_t>(mx, (int64_t)B * d);
  float *G0 = (float *)net->grads.ptr, *G1 = G0 + mx;
  const unsigned nbl = cdiv(cnt, 256);
  mse_grad_kernel<<<nbl, 256, 0, st>>>(cnt, 1.f / (float)cnt, acts + net->act_off(L, B), T, G0, (double *)net->part.ptr);
  sum_parts_kernel<<<1, 32, 0, st>>>((int)nbl, (const double *)net->part.ptr, 1.0 / (double)cnt, (double *)net->loss.ptr);
  // backward: G0 holds dLoss/dZ_l (pre-activation) of layer l
  for (int l = L - 1; l >= 0; --l) {
    const int K = net->dims[l], N = net->dims[l + 1];
    const float *Yin = l == 0 ? X : acts + net->act_off(l, B);
    // dW_l[n, k] = sum_b G[b, n] Yin[b, k]
    gemm<float>(st, N, K, B, G0, 1, N, Yin, K, 1, g + net->woff[l], K, EPI_NONE, nullptr, nullptr);
    colsum_kernel<<<cdiv(N, 128), 128, 0, st>>>(B, N, G0, g + net->boff[l]);
    if (l > 0) {
      // dZ_{l-1}[b, k] = (sum_n G[b, n] W[n, k]) * (1 - Yin[b, k]^2)
      gemm<__nv_bfloat16>(st, B, K, N, G0, N, 1, wb + net->woff[l], K, 1, G1, K, EPI_TANH_GRAD, nullptr, Yin);
      std::swap(G0, G1);
    }
  }
  MLP_CK(cudaGetLastError());
  if (grads_host) {
    MLP_CK(cudaMemcpyAsync(grads_host, g, 4 * net->n_params, cudaMemcpyDeviceToHost, st));
  }
  if (loss_host) {
    MLP_CK(cudaMemcpyAsync(loss_host, net->loss.ptr, 8, cudaMemcpyDeviceToHost, st));
  }
  if (lr > 0.f) {
    ++net->steps;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - (float)std::pow(b1, (double)net->steps), c2 = 1.f - (float)std::pow(b2, (double)net->steps);
    adam_kernel<<<cdiv(net->n_params, 256), 256, 0, st>>>(net->n_params, (float *)net->w.ptr, g, (float *)net->m.ptr,
                                                          (float *)net->v.ptr, (__nv_bfloat16 *)net->wb.ptr, lr, b1,
                                                          b2, 1e-8f, c1, c2);
    MLP_CK(cudaGetLastError());
  }
  if (loss_host || grads_host) MLP_CK(cudaStreamSynchronize(st));
  return MBC_OK;
}
