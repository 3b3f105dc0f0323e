// ref_driver.cpp -- drives the REFERENCE's own host code for parity pinning.
// TEST INFRASTRUCTURE ONLY; built by oracle/Makefile into oracle/_ref/.
//
// It includes the reference's src/maxmin.h (heap ordering create_ordering_3d)
// and src/nanoflann.hpp (kd-tree) from the reference tree, unmodified, and
// exposes two C entry points:
//   ref_order   -- fps_sampler::fast_fps (preprocess.h:782-831) around the
//                  reference's create_ordering_3d (maxmin.h:588-665).
//   ref_pattern -- fps_sampler::simpl_sparsity (preprocess.h:235-316) using the
//                  reference's nanoflann radiusSearch with leaf size 10
//                  (preprocess.h:24-28) below the cutoff, brute force above.
// The few lines of preprocess.h that wrap these calls use Eigen, which cannot
// be built here, so they are restated (same predicates, same arithmetic).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <memory>
#include <utility>
#include <vector>

#include "maxmin.h"

namespace {

double sqnorm_rows(const double *a, const double *b)
{
  const double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
  return (dx * dx + dy * dy) + dz * dz;
}

}  // namespace

extern "C" int ref_order(int n, const double *pts, int32_t *P, double *scale)
{
  if (n <= 0) return 1;
  // preprocess.h:786-814
  double corner[3] = {pts[0], pts[1], pts[2]};
  for (int k = 1; k < n; ++k)
    for (int d = 0; d < 3; ++d) corner[d] = std::min(corner[d], pts[3 * k + d]);
  int first_idx = -1;
  double best = 1e10;
  for (int i = 0; i < n; ++i) {
    const double d = sqnorm_rows(&pts[3 * i], corner);
    if (d < best) {
      best = d;
      first_idx = i;
    }
  }
  if (first_idx < 0) return 1;
  std::vector<unsigned int> seq(n), rev_seq(n);
  std::vector<double> dists(n);
  seq[0] = first_idx;
  create_ordering_3d(&seq[0], &rev_seq[0], dists.data(), n, pts, first_idx, nullptr);
  for (int i = 0; i < n; ++i) P[i] = -1;
  for (int i = 0; i < n; ++i) {
    if (P[seq[i]] != -1) return 3;
    P[seq[i]] = n - 1 - i;
    scale[n - 1 - i] = dists[i];
  }
  return 0;
}

// pts: ORIGINAL order; P, scale from ref_order.  Count pass when ind == NULL.
extern "C" int64_t ref_pattern(int n, const double *pts, const int32_t *P, const double *scale,
                               double rho, int32_t *ptr, int32_t *ind)
{
  klchol::RmMatF_t M(n, 3);
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) M(i, d) = pts[3 * i + d];
  KDTree kdt(3, std::cref(M), 10);
  std::vector<int32_t> Pinv(n);
  for (int i = 0; i < n; ++i) Pinv[P[i]] = i;

  double cutoff = 0.5;
  if (rho <= 2.0) cutoff = 0.95;
  else if (rho >= 7) cutoff = 0.75;
  else cutoff = -0.04 * rho + 1.03;

  std::vector<std::vector<int32_t>> nei(n);
#pragma omp parallel for schedule(dynamic, 64)
  for (int j = 0; j < n; ++j) {
    const int J = Pinv[j];
    const double lj = rho * scale[j];
    if (1.0 * j < cutoff * n) {
      std::vector<std::pair<long int, double>> matches;
      kdt.index->radiusSearch(&M(J, 0), lj * lj, matches, nanoflann::SearchParams());
      for (const auto &res : matches) {
        const int i = P[res.first];
        const int I = (int)res.first;
        const double li = rho * scale[i];
        if (i >= j && sqnorm_rows(&pts[3 * I], &pts[3 * J]) < std::min(li * li, lj * lj))
          nei[j].push_back(i);
      }
    } else {
      for (int i = j; i < n; ++i) {
        const int I = Pinv[i];
        const double li = rho * scale[i];
        if (sqnorm_rows(&pts[3 * I], &pts[3 * J]) < std::min(li * li, lj * lj)) nei[j].push_back(i);
      }
    }
  }
  int64_t total = 0;
  ptr[0] = 0;
  for (int j = 0; j < n; ++j) {
    total += (int64_t)nei[j].size();
    ptr[j + 1] = (int32_t)total;
  }
  if (ind) {
    for (int j = 0; j < n; ++j) {
      std::sort(nei[j].begin(), nei[j].end());
      std::copy(nei[j].begin(), nei[j].end(), ind + ptr[j]);
    }
  }
  return total;
}
