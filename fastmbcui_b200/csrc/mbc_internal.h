// Internal declarations shared by the host plan and the CUDA solver.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "mbc.h"

namespace mbc {

// Thread-local error message behind mbc_last_error().
void set_error(const std::string &msg);
mbc_status fail(mbc_status s, const std::string &msg);

// Host plan: everything the factor and PCG need that is integer work.
struct Plan {
  int32_t n = 0;
  double rho = 3.0, lambda = 1.5;
  int32_t max_super = 2048;
  int32_t root = -1;
  std::vector<double> pts;       // original order, n x 3
  std::vector<int32_t> P, Pinv;  // P[orig] = new, Pinv[new] = orig
  std::vector<double> scale;     // new order, ascending
  std::vector<int32_t> ptr, ind; // MRA pattern (CSC, new order)
  std::vector<int32_t> sup_ptr, sup_ind, sup_parent;
  std::vector<int32_t> set_ptr, set_ind;  // supernode row sets (sorted)
  std::vector<int32_t> lptr, lind;        // factor pattern (CSC)
  std::vector<int64_t> th_ptr;            // Theta offsets, n_s^2 per supernode
  // Row-wise view of the factor: for row i, entries k of L with lind[k] == i,
  // as (column, value index) pairs; used for the gather form of z = L u.
  std::vector<int32_t> rptr, rcol, rmap;
  int32_t n_super = 0, max_set = 0;
  double t_order_ms = 0, t_pattern_ms = 0, t_super_ms = 0;
};

// Maximin ordering (maxmin.h:588-665 + preprocess.h:782-831).
mbc_status build_order(Plan &p, int n_threads);
// MRA pattern (preprocess.h:235-316).
mbc_status build_pattern(Plan &p, int n_threads);
// Supernodes and their row sets (preprocess.h:541-671).
mbc_status build_supernodes(Plan &p, int n_threads);
// Morton (Z-curve) order of n points with coordinates at pts[i * stride + 0..2]
// (mbc_spatial_order).
mbc_status spatial_order(int32_t n, const float *pts, int32_t stride, int32_t *order);

}  // namespace mbc

struct mbc_plan {
  mbc::Plan p;
};
