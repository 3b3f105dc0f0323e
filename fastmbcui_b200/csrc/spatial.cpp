// Spatially coherent orders of point sets (host).
//
// The FP64-accurate INT8 matvec scales its operand by a power of two per
// (output row, 2048-wide chunk of the reduction axis).  A chunk that holds
// points from all over the scene holds near-field entries for every output
// row, so every chunk's scale is set by the near field and the far field
// keeps few bits.  Walking the reduction axis in Morton (Z-curve) order makes
// each chunk a compact region: only the few chunks near an output row carry
// its near field, and the rest are scaled to their own far-field values.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "mbc_internal.h"

namespace mbc {

namespace {

// spread the low 21 bits of v to every third bit
inline uint64_t spread3(uint64_t v)
{
  v &= 0x1FFFFF;
  v = (v | (v << 32)) & 0x1F00000000FFFFull;
  v = (v | (v << 16)) & 0x1F0000FF0000FFull;
  v = (v | (v << 8)) & 0x100F00F00F00F00Full;
  v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
  v = (v | (v << 2)) & 0x1249249249249249ull;
  return v;
}

}  // namespace

mbc_status spatial_order(int32_t n, const float *pts, int32_t stride, int32_t *order)
{
  if (n < 0 || (n > 0 && (!pts || !order)) || stride < 3) return fail(MBC_BAD_ARG, "spatial order: bad arguments");
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int32_t i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) {
      const double v = pts[(size_t)i * stride + d];
      if (!std::isfinite(v)) return fail(MBC_BAD_ARG, "spatial order: non-finite coordinate");
      lo[d] = std::min(lo[d], v);
      hi[d] = std::max(hi[d], v);
    }
  // one cube for all axes, so the curve's cells stay cubes
  double ext = 0.0;
  for (int d = 0; d < 3; ++d) ext = std::max(ext, hi[d] - lo[d]);
  const double scale = ext > 0.0 ? (double)((1u << 21) - 1) / ext : 0.0;
  std::vector<std::pair<uint64_t, int32_t>> key((size_t)n);
  for (int32_t i = 0; i < n; ++i) {
    uint64_t c = 0;
    for (int d = 0; d < 3; ++d) {
      double q = std::floor((pts[(size_t)i * stride + d] - lo[d]) * scale);
      q = std::min(std::max(q, 0.0), (double)((1u << 21) - 1));
      c |= spread3((uint64_t)q) << (2 - d);
    }
    key[(size_t)i] = {c, i};
  }
  std::sort(key.begin(), key.end());  // ties by index
  for (int32_t i = 0; i < n; ++i) order[i] = key[(size_t)i].second;
  return MBC_OK;
}

}  // namespace mbc

extern "C" mbc_status mbc_spatial_order(int32_t n, const float *pts_host, int32_t stride, int32_t *order_host)
{
  return mbc::spatial_order(n, pts_host, stride, order_host);
}
