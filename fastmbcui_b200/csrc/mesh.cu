// mesh.cu -- the mesh collocation operator assembled on the device.
//
// The reference builds the collocation matrix of a triangle-mesh scene in
// torch every step (core/KTAB_Mfs_spclf1d.py:95-113): the solid angle of every
// face seen from every source (utils/torch_utils.py:306-334,
// compute_solid_angle, through faces x sources x 3 temporaries) and the
// rigid-mode right-hand side FL @ IQ (compute_FL_matrix, :62-75, and
// compute_face_centers, :49-60).  Here one thread computes one entry in FP64
// from float32 coordinates and stores it as FP32 or FP64, with no temporaries.
#include <cmath>
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "mbc_internal.h"

namespace {

template <typename T>
__device__ __forceinline__ T to_out(double v);
template <>
__device__ __forceinline__ float to_out<float>(double v) { return (float)v; }
template <>
__device__ __forceinline__ double to_out<double>(double v) { return v; }

// M[f, j] = 2 atan2(R1 . (R2 x R3), l1 l2 l3 + (R1.R2) l3 + (R1.R3) l2 + (R2.R3) l1),
// Rk = V[F[f, k]] - S[j] (van Oosterom and Strackee).  Block: 128 sources of
// one face; faces loop over gridDim.y so any face count fits the grid.
template <typename T>
__global__ void __launch_bounds__(128) solid_angle_kernel(int n_vert, const float *__restrict__ V, int n_faces,
                                                          const int32_t *__restrict__ F, int n_src,
                                                          const float *__restrict__ S, T *__restrict__ M,
                                                          int64_t ldm)
{
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_src) return;
  const double sx = S[3 * (size_t)j], sy = S[3 * (size_t)j + 1], sz = S[3 * (size_t)j + 2];
  for (int f = blockIdx.y; f < n_faces; f += gridDim.y) {
    const int i1 = F[3 * (size_t)f], i2 = F[3 * (size_t)f + 1], i3 = F[3 * (size_t)f + 2];
    double out;
    if (i1 < 0 || i1 >= n_vert || i2 < 0 || i2 >= n_vert || i3 < 0 || i3 >= n_vert) {
      out = nan("");  // a face naming a vertex that does not exist
    } else {
      const double ax = V[3 * (size_t)i1] - sx, ay = V[3 * (size_t)i1 + 1] - sy, az = V[3 * (size_t)i1 + 2] - sz;
      const double bx = V[3 * (size_t)i2] - sx, by = V[3 * (size_t)i2 + 1] - sy, bz = V[3 * (size_t)i2 + 2] - sz;
      const double cx = V[3 * (size_t)i3] - sx, cy = V[3 * (size_t)i3 + 1] - sy, cz = V[3 * (size_t)i3 + 2] - sz;
      const double num = ax * (by * cz - bz * cy) + ay * (bz * cx - bx * cz) + az * (bx * cy - by * cx);
      const double la = sqrt(ax * ax + ay * ay + az * az);
      const double lb = sqrt(bx * bx + by * by + bz * bz);
      const double lc = sqrt(cx * cx + cy * cy + cz * cz);
      const double ab = ax * bx + ay * by + az * bz;
      const double ac = ax * cx + ay * cy + az * cz;
      const double bc = bx * cx + by * cy + bz * cz;
      out = 2.0 * atan2(num, la * lb * lc + ab * lc + ac * lb + bc * la);
    }
    M[(size_t)f * ldm + j] = to_out<T>(out);
  }
}

// rhs[f, 6b .. 6b+5] = (s, r x s) for the face's body b, zero elsewhere:
// s = (v2 - v1) x (v3 - v1) / 2, r = (v1 + v2 + v3) / 3 - y_b.  One thread
// per face writes its whole row (6 n_bodies entries).
template <typename T>
__global__ void rhs_kernel(int n_vert, const float *__restrict__ V, int n_faces, const int32_t *__restrict__ F,
                           const int32_t *__restrict__ face_body, int n_bodies, const float *__restrict__ body_pos,
                           T *__restrict__ rhs)
{
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n_faces) return;
  const int ncol = 6 * n_bodies;
  T *row = rhs + (size_t)f * ncol;
  const int i1 = F[3 * (size_t)f], i2 = F[3 * (size_t)f + 1], i3 = F[3 * (size_t)f + 2];
  const int b = face_body[f];
  if (i1 < 0 || i1 >= n_vert || i2 < 0 || i2 >= n_vert || i3 < 0 || i3 >= n_vert || b < 0 || b >= n_bodies) {
    for (int c = 0; c < ncol; ++c) row[c] = to_out<T>(nan(""));
    return;
  }
  for (int c = 0; c < ncol; ++c) row[c] = to_out<T>(0.0);
  const double v1x = V[3 * (size_t)i1], v1y = V[3 * (size_t)i1 + 1], v1z = V[3 * (size_t)i1 + 2];
  const double v2x = V[3 * (size_t)i2], v2y = V[3 * (size_t)i2 + 1], v2z = V[3 * (size_t)i2 + 2];
  const double v3x = V[3 * (size_t)i3], v3y = V[3 * (size_t)i3 + 1], v3z = V[3 * (size_t)i3 + 2];
  const double e1x = v2x - v1x, e1y = v2y - v1y, e1z = v2z - v1z;
  const double e2x = v3x - v1x, e2y = v3y - v1y, e2z = v3z - v1z;
  const double sx = (e1y * e2z - e1z * e2y) / 2.0, sy = (e1z * e2x - e1x * e2z) / 2.0,
               sz = (e1x * e2y - e1y * e2x) / 2.0;
  const double rx = (v1x + v2x + v3x) / 3.0 - body_pos[3 * b];
  const double ry = (v1y + v2y + v3y) / 3.0 - body_pos[3 * b + 1];
  const double rz = (v1z + v2z + v3z) / 3.0 - body_pos[3 * b + 2];
  T *o = row + 6 * b;
  o[0] = to_out<T>(sx);
  o[1] = to_out<T>(sy);
  o[2] = to_out<T>(sz);
  o[3] = to_out<T>(ry * sz - rz * sy);
  o[4] = to_out<T>(rz * sx - rx * sz);
  o[5] = to_out<T>(rx * sy - ry * sx);
}

template <typename T>
void launch(int32_t n_vert, const float *V, int32_t n_faces, const int32_t *F, const int32_t *face_body,
            int32_t n_bodies, const float *body_pos, int32_t n_src, const float *S, void *M, int64_t ldm, void *rhs,
            cudaStream_t st)
{
  const dim3 grid((unsigned)((n_src + 127) / 128), (unsigned)(n_faces < 65535 ? n_faces : 65535));
  solid_angle_kernel<T><<<grid, 128, 0, st>>>(n_vert, V, n_faces, F, n_src, S, (T *)M, ldm);
  if (rhs)
    rhs_kernel<T><<<(unsigned)((n_faces + 127) / 128), 128, 0, st>>>(n_vert, V, n_faces, F, face_body, n_bodies,
                                                                       body_pos, (T *)rhs);
}

}  // namespace

extern "C" mbc_status mbc_mesh_assemble(int32_t n_vert, const float *V, int32_t n_faces, const int32_t *F,
                                        const int32_t *face_body, int32_t n_bodies, const float *body_pos,
                                        int32_t n_src, const float *S, int32_t dtype, void *M, int64_t ldm,
                                        void *rhs, mbc_stream stream)
{
  if (n_vert <= 0 || n_faces <= 0 || n_src <= 0 || !V || !F || !S || !M)
    return mbc::fail(MBC_BAD_ARG, "mbc_mesh_assemble: NULL pointer or non-positive size");
  if (ldm < n_src) return mbc::fail(MBC_BAD_ARG, "mbc_mesh_assemble: ldm below n_src");
  if (dtype != MBC_F32 && dtype != MBC_F64) return mbc::fail(MBC_BAD_ARG, "mbc_mesh_assemble: dtype must be MBC_F32 or MBC_F64");
  if (rhs && (n_bodies <= 0 || !face_body || !body_pos))
    return mbc::fail(MBC_BAD_ARG, "mbc_mesh_assemble: the right-hand side needs face_body, n_bodies and body_pos");
  const cudaStream_t st = (cudaStream_t)stream;
  if (dtype == MBC_F64)
    launch<double>(n_vert, V, n_faces, F, face_body, n_bodies, body_pos, n_src, S, M, ldm, rhs, st);
  else
    launch<float>(n_vert, V, n_faces, F, face_body, n_bodies, body_pos, n_src, S, M, ldm, rhs, st);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return mbc::fail(MBC_CUDA_ERROR, std::string("mbc_mesh_assemble: ") + cudaGetErrorString(e));
  return MBC_OK;
}
