// Host plan for the MFS solve path: maximin ordering, MRA sparsity pattern,
// greedy supernodes and the supernodal factor pattern.
//
// All of it is integer / comparison work whose result must equal the
// reference bit for bit, so every distance is computed as
//   d2 = (dx*dx + dy*dy) + dz*dz
// with separately rounded products (the file is built with -ffp-contract=off),
// which is the value src/maxmin.h:370-374, Eigen's squaredNorm of a 3-vector
// and nanoflann's L2_Adaptor all produce.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <new>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "mbc_internal.h"

namespace mbc {

namespace {

thread_local std::string g_last_error;

inline double sq3(const double *a, const double *b)
{
  const double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
  return (dx * dx + dy * dy) + dz * dz;
}

double ms_since(std::chrono::steady_clock::time_point t0)
{
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// Max-heap over point ids keyed by the distance to the selected set, with
// the reference's semantics: fixed implicit tree (children 2k+1, 2k+2),
// initial keys 10000 for nodes with two children and +inf otherwise
// (maxmin.h:274-293), and updates that only sift down (maxmin.h:194-271).
struct SiftDownHeap {
  std::vector<double> key;
  std::vector<int32_t> id, slot;
  int32_t n;

  explicit SiftDownHeap(int32_t n_) : key(n_), id(n_), slot(n_), n(n_)
  {
    for (int32_t k = 0; k < n; ++k) {
      key[k] = (2 * (int64_t)k + 2 < n) ? 10000.0 : std::numeric_limits<double>::infinity();
      id[k] = k;
      slot[k] = k;
    }
  }

  void set(int32_t point, double d)
  {
    int32_t a = slot[point];
    key[a] = d;
    for (;;) {
      const int64_t l = 2 * (int64_t)a + 1, r = l + 1;
      int32_t c;
      if (l >= n) return;
      if (r >= n) {
        if (!(key[a] < key[l])) return;
        c = (int32_t)l;
      } else if (key[l] > key[r]) {
        if (!(key[a] < key[l])) return;
        c = (int32_t)l;
      } else {
        if (!(key[a] < key[r])) return;
        c = (int32_t)r;
      }
      std::swap(key[a], key[c]);
      std::swap(id[a], id[c]);
      slot[id[a]] = a;
      slot[id[c]] = c;
      a = c;
    }
  }
  double get(int32_t point) const { return key[slot[point]]; }
};

}  // namespace

void set_error(const std::string &msg) { g_last_error = msg; }
mbc_status fail(mbc_status s, const std::string &msg)
{
  g_last_error = msg;
  return s;
}
const char *last_error_cstr() { return g_last_error.c_str(); }

// candidate lists at least this long are filtered by several threads
constexpr int32_t kParallelScan = 4096;

mbc_status build_order(Plan &p, int n_threads)
{
  const auto t0 = std::chrono::steady_clock::now();
  const int32_t n = p.n;
  const double *x = p.pts.data();
  // root: first point strictly closest to the column-wise minimum corner,
  // starting from 1e10 (preprocess.h:786-814)
  double corner[3] = {x[0], x[1], x[2]};
  for (int32_t k = 1; k < n; ++k)
    for (int d = 0; d < 3; ++d) corner[d] = std::min(corner[d], x[3 * k + d]);
  int32_t root = -1;
  double best = 1e10;
  for (int32_t k = 0; k < n; ++k) {
    const double d = sq3(&x[3 * k], corner);
    if (d < best) {
      best = d;
      root = k;
    }
  }
  if (root < 0) return fail(MBC_BAD_ARG, "no point within 1e5 of the bounding-box corner");
  p.root = root;

  // create_ordering_3d (maxmin.h:588-665) without a boundary (dist_bd = 1e16)
  SiftDownHeap heap(n);
  std::vector<int32_t> seq(n), parent(n, 0), li(n + 1, 0), lj;
  std::vector<double> dist(n);
  lj.reserve((size_t)n * 8);
  seq[0] = root;
  dist[0] = 0.0;
  for (int32_t k = 0; k < n; ++k) {
    const double d = std::sqrt(sq3(&x[3 * root], &x[3 * k]));
    lj.push_back(k);
    if (d > dist[0]) dist[0] = d;
    heap.set(k, std::min(d, 1e16));
  }
  li[1] = n;
  // The early pivots scan long candidate lists (their parent is the root,
  // whose list holds every point) of which few pass the distance test: at
  // N = 64000, 72 % of the 31 M tests fall in lists of 4096 or more and 4 %
  // pass.  The test depends only on the pivot, so a long list is filtered
  // by several threads, each keeping its hits in list order, and the hits
  // are then visited in list order exactly as the serial loop does: the
  // heap updates, the appended children and the parents are the same.
#ifdef _OPENMP
  const int nthr = n_threads > 0 ? n_threads : omp_get_max_threads();
#else
  const int nthr = 1;
  (void)n_threads;
#endif
  std::vector<std::vector<std::pair<int32_t, double>>> hits(nthr);
  for (int32_t k = 1; k < n; ++k) {
    const int32_t piv = heap.id[0];
    const double pd = heap.key[0];
    seq[k] = piv;
    dist[k] = pd;
    const int32_t kmin = li[parent[piv]], kmax = li[parent[piv] + 1];
    li[k + 1] = li[k];
    const double *xp = &x[3 * piv];
    const double pd2 = pd * pd;
    auto visit = [&](int32_t j, double t2) {
      const double t = std::sqrt(t2);  // the same value at both uses below
      double jd = heap.get(j);
      if (t2 < jd * jd) {
        const double nd = std::min(t, 1e16);
        heap.set(j, nd);
        jd = nd;
      }
      lj.push_back(j);
      ++li[k + 1];
      if (t + jd < pd) parent[j] = k;
    };
    if (nthr > 1 && kmax - kmin >= kParallelScan) {
      for (auto &h : hits) h.clear();
#ifdef _OPENMP
#pragma omp parallel num_threads(nthr)
      {
        const int t = omp_get_thread_num(), nt = omp_get_num_threads();
        const int64_t len = kmax - kmin;
        const int32_t b = kmin + (int32_t)(len * t / nt), e = kmin + (int32_t)(len * (t + 1) / nt);
        auto &h = hits[t];
        for (int32_t kk = b; kk < e; ++kk) {
          const int32_t j = lj[kk];
          const double t2 = sq3(xp, &x[3 * j]);
          if (t2 < pd2) h.emplace_back(j, t2);
        }
      }
#endif
      for (const auto &h : hits)
        for (const auto &jt : h) visit(jt.first, jt.second);
    } else {
      for (int32_t kk = kmin; kk < kmax; ++kk) {
        const int32_t j = lj[kk];
        const double t2 = sq3(xp, &x[3 * j]);
        if (t2 < pd2) visit(j, t2);
      }
    }
  }
  // fine-to-coarse: P[seq[i]] = n-1-i, scale reversed (preprocess.h:825-830)
  p.P.assign(n, -1);
  p.Pinv.assign(n, 0);
  p.scale.assign(n, 0.0);
  for (int32_t i = 0; i < n; ++i) {
    if (p.P[seq[i]] != -1) return fail(MBC_COVERAGE, "maximin ordering is not a permutation");
    p.P[seq[i]] = n - 1 - i;
    p.Pinv[n - 1 - i] = seq[i];
    p.scale[n - 1 - i] = dist[i];
  }
  // preprocess.h:74-77 asserts ascending length scales
  for (int32_t i = 1; i < n; ++i)
    if (p.scale[i] < p.scale[i - 1])
      return fail(MBC_BAD_ARG, "length scales are not ascending (degenerate point set)");
  p.t_order_ms = ms_since(t0);
  return MBC_OK;
}

namespace {

// Uniform grid over the points (new order) for radius queries.
struct Grid {
  double lo[3], h;
  int32_t dim[3];
  std::vector<int32_t> start, items;  // items sorted by cell

  void build(const std::vector<double> &q, int32_t n)
  {
    double hi[3];
    for (int d = 0; d < 3; ++d) lo[d] = hi[d] = q[d];
    for (int32_t i = 1; i < n; ++i)
      for (int d = 0; d < 3; ++d) {
        lo[d] = std::min(lo[d], q[3 * i + d]);
        hi[d] = std::max(hi[d], q[3 * i + d]);
      }
    double ext = 0;
    for (int d = 0; d < 3; ++d) ext = std::max(ext, hi[d] - lo[d]);
    // ~2 points per occupied cell on a surface: cells ~ n^(3/2) / 2 is too
    // many; aim at n/2 cells over the bounding box instead.
    double vol = 1.0;
    for (int d = 0; d < 3; ++d) vol *= std::max(hi[d] - lo[d], ext * 1e-3);
    h = std::cbrt(vol / std::max(1.0, n / 2.0));
    if (!(h > 0)) h = 1.0;
    int64_t cells = 1;
    for (int d = 0; d < 3; ++d) {
      dim[d] = std::max<int32_t>(1, (int32_t)std::floor((hi[d] - lo[d]) / h) + 1);
      cells *= dim[d];
    }
    while (cells > 4LL * n + 64) {  // guard against degenerate extents
      h *= 1.25;
      cells = 1;
      for (int d = 0; d < 3; ++d) {
        dim[d] = std::max<int32_t>(1, (int32_t)std::floor((hi[d] - lo[d]) / h) + 1);
        cells *= dim[d];
      }
    }
    start.assign(cells + 1, 0);
    std::vector<int32_t> cell(n);
    for (int32_t i = 0; i < n; ++i) {
      cell[i] = cell_of(&q[3 * i]);
      ++start[cell[i] + 1];
    }
    for (int64_t c = 0; c < cells; ++c) start[c + 1] += start[c];
    items.resize(n);
    std::vector<int32_t> fill(start.begin(), start.end() - 1);
    for (int32_t i = 0; i < n; ++i) items[fill[cell[i]]++] = i;  // ascending i within a cell
  }
  int32_t coord(double v, int d) const
  {
    const double c = std::floor((v - lo[d]) / h);
    if (c < 0) return 0;
    if (c >= dim[d]) return dim[d] - 1;
    return (int32_t)c;
  }
  int32_t cell_of(const double *v) const
  {
    return (coord(v[2], 2) * dim[1] + coord(v[1], 1)) * dim[0] + coord(v[0], 0);
  }
};

}  // namespace

mbc_status build_pattern(Plan &p, int n_threads)
{
  const auto t0 = std::chrono::steady_clock::now();
  const int32_t n = p.n;
  const double rho = p.rho;
  // points in the new order
  std::vector<double> q((size_t)3 * n);
  for (int32_t i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) q[3 * i + d] = p.pts[3 * (size_t)p.Pinv[i] + d];
  Grid g;
  g.build(q, n);
  const int64_t cells = (int64_t)g.dim[0] * g.dim[1] * g.dim[2];

  std::vector<std::vector<int32_t>> nei(n);
#ifdef _OPENMP
  const int nt = n_threads > 0 ? n_threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 32) num_threads(nt)
#else
  (void)n_threads;
#endif
  for (int32_t j = 0; j < n; ++j) {
    const double lj = rho * p.scale[j];
    const double lj2 = lj * lj;
    const double *xj = &q[3 * (size_t)j];
    auto &out = nei[j];
    // cell box covering the ball of radius lj, widened by one cell so that
    // rounding in the cell coordinates can never drop a candidate
    int32_t c0[3], c1[3];
    int64_t box = 1;
    for (int d = 0; d < 3; ++d) {
      c0[d] = std::max(0, g.coord(xj[d] - lj, d) - 1);
      c1[d] = std::min(g.dim[d] - 1, g.coord(xj[d] + lj, d) + 1);
      box *= (int64_t)(c1[d] - c0[d] + 1);
    }
    if (box * 4 > cells || box > (int64_t)(n - j)) {
      for (int32_t i = j; i < n; ++i) {
        const double li = rho * p.scale[i];
        if (sq3(&q[3 * (size_t)i], xj) < std::min(li * li, lj2)) out.push_back(i);
      }
    } else {
      for (int32_t cz = c0[2]; cz <= c1[2]; ++cz)
        for (int32_t cy = c0[1]; cy <= c1[1]; ++cy) {
          const int64_t rowc = ((int64_t)cz * g.dim[1] + cy) * g.dim[0];
          const int32_t b = g.start[rowc + c0[0]], e = g.start[rowc + c1[0] + 1];
          for (int32_t t = b; t < e; ++t) {
            const int32_t i = g.items[t];
            if (i < j) continue;
            const double li = rho * p.scale[i];
            if (sq3(&q[3 * (size_t)i], xj) < std::min(li * li, lj2)) out.push_back(i);
          }
        }
      std::sort(out.begin(), out.end());
    }
  }
  p.ptr.assign(n + 1, 0);
  for (int32_t j = 0; j < n; ++j) {
    const int64_t next = (int64_t)p.ptr[j] + (int64_t)nei[j].size();
    if (next > std::numeric_limits<int32_t>::max())
      return fail(MBC_NO_MEMORY, "pattern has more than 2^31 entries");
    p.ptr[j + 1] = (int32_t)next;
  }
  p.ind.resize(p.ptr[n]);
  for (int32_t j = 0; j < n; ++j) std::copy(nei[j].begin(), nei[j].end(), p.ind.begin() + p.ptr[j]);
  p.t_pattern_ms = ms_since(t0);
  return MBC_OK;
}

namespace {

// Transpose of an n-column CSC pattern (ptr, ind): row i of the result lists
// its columns in ascending order, with map[t] = the position in ind of that
// entry (optional), exactly what a serial counting sort over ascending
// columns gives.  Threads take contiguous column chunks of about equal
// entries, count their rows, and fill them in column order at offsets that
// place chunk t's entries of a row after those of chunks 0 .. t-1.
void transpose_csc(int32_t n, const std::vector<int32_t> &ptr, const std::vector<int32_t> &ind,
                   std::vector<int32_t> &tptr, std::vector<int32_t> &tind, std::vector<int32_t> *map,
                   int n_threads)
{
  const int64_t nnz = ptr[n];
  int want = 1;
#ifdef _OPENMP
  want = n_threads > 0 ? n_threads : omp_get_max_threads();
#else
  (void)n_threads;
#endif
  want = (int)std::max<int64_t>(1, std::min<int64_t>(want, nnz / 65536));
  std::vector<int32_t> c0;   // column chunk bounds, one chunk per thread of the team
  std::vector<int32_t> cnt;  // per chunk: entries of row i, then its write offset
  tptr.assign(n + 1, 0);
  tind.resize(nnz);
  if (map) map->resize(nnz);
  int nt = 1;
#pragma omp parallel num_threads(want)
  {
    int t = 0;
#ifdef _OPENMP
    t = omp_get_thread_num();
#endif
#pragma omp single
    {
#ifdef _OPENMP
      nt = omp_get_num_threads();  // the team actually granted
#endif
      c0.assign(nt + 1, n);
      c0[0] = 0;
      for (int u = 1; u < nt; ++u)
        c0[u] = (int32_t)(std::lower_bound(ptr.begin(), ptr.begin() + n + 1, (int32_t)(nnz * u / nt)) -
                          ptr.begin());
      cnt.assign((size_t)nt * (n + 1), 0);
    }
    int32_t *c = cnt.data() + (size_t)t * (n + 1);
    for (int32_t j = c0[t]; j < c0[t + 1]; ++j)
      for (int32_t k = ptr[j]; k < ptr[j + 1]; ++k) ++c[ind[k]];
#pragma omp barrier
#pragma omp for schedule(static)
    for (int32_t i = 0; i < n; ++i) {
      int32_t tot = 0;
      for (int u = 0; u < nt; ++u) tot += cnt[(size_t)u * (n + 1) + i];
      tptr[i + 1] = tot;
    }
#pragma omp single
    for (int32_t i = 0; i < n; ++i) tptr[i + 1] += tptr[i];
#pragma omp for schedule(static)
    for (int32_t i = 0; i < n; ++i) {
      int32_t off = tptr[i];
      for (int u = 0; u < nt; ++u) {
        int32_t &e = cnt[(size_t)u * (n + 1) + i];
        const int32_t m = e;
        e = off;
        off += m;
      }
    }
    for (int32_t j = c0[t]; j < c0[t + 1]; ++j)
      for (int32_t k = ptr[j]; k < ptr[j + 1]; ++k) {
        const int32_t q = c[ind[k]]++;
        tind[q] = j;
        if (map) (*map)[q] = k;
      }
  }
}

}  // namespace

mbc_status build_supernodes(Plan &p, int n_threads)
{
  const auto t0 = std::chrono::steady_clock::now();
  const int32_t n = p.n;
  // aggregate (preprocess.h:541-602), dim 1 and one group {0, n}
  std::vector<unsigned char> vis(n, 0);
  p.sup_ptr.assign(1, 0);
  p.sup_ind.resize(n);
  p.sup_parent.assign(n, -1);
  int32_t pos = 0, ns = 0;
  for (int32_t j = 0; j < n; ++j) {
    if (vis[j]) continue;
    int32_t size = 0;
    const double lim = p.lambda * p.scale[j];
    for (int32_t k = p.ptr[j]; k < p.ptr[j + 1]; ++k) {
      const int32_t i = p.ind[k];
      if (!vis[i] && p.scale[i] <= lim) {
        vis[i] = 1;
        p.sup_ind[pos++] = i;
        p.sup_parent[i] = ns;
        if (++size >= p.max_super) break;
      }
    }
    ++ns;
    p.sup_ptr.push_back(pos);
  }
  if (pos != n) return fail(MBC_COVERAGE, "aggregation did not cover every point (duplicate points?)");
  p.n_super = ns;

  // super_sparsity (preprocess.h:604-671): the row set of a supernode is the
  // sorted union of its columns' rows.  Walking rows i ascending and the
  // columns J of row i (the transpose) appends i at most once per supernode.
  std::vector<int32_t> tptr, tind;
  transpose_csc(n, p.ptr, p.ind, tptr, tind, nullptr, n_threads);
  std::vector<int32_t> last(ns, -1), cnt(ns, 0);
  for (int32_t i = 0; i < n; ++i)
    for (int32_t k = tptr[i]; k < tptr[i + 1]; ++k) {
      const int32_t s = p.sup_parent[tind[k]];
      if (last[s] != i) {
        last[s] = i;
        ++cnt[s];
      }
    }
  p.set_ptr.assign(ns + 1, 0);
  for (int32_t s = 0; s < ns; ++s) p.set_ptr[s + 1] = p.set_ptr[s] + cnt[s];
  p.set_ind.resize(p.set_ptr[ns]);
  std::fill(last.begin(), last.end(), -1);
  std::vector<int32_t> wpos(p.set_ptr.begin(), p.set_ptr.end() - 1);
  for (int32_t i = 0; i < n; ++i)
    for (int32_t k = tptr[i]; k < tptr[i + 1]; ++k) {
      const int32_t s = p.sup_parent[tind[k]];
      if (last[s] != i) {
        last[s] = i;
        p.set_ind[wpos[s]++] = i;
      }
    }
  // column j keeps the suffix >= j of its supernode's row set
  p.lptr.assign(n + 1, 0);
  std::vector<int32_t> off(n);
  for (int32_t j = 0; j < n; ++j) {
    const int32_t s = p.sup_parent[j];
    const auto b = p.set_ind.begin() + p.set_ptr[s], e = p.set_ind.begin() + p.set_ptr[s + 1];
    off[j] = (int32_t)(std::lower_bound(b, e, j) - p.set_ind.begin());
    const int64_t next = (int64_t)p.lptr[j] + (p.set_ptr[s + 1] - off[j]);
    if (next > std::numeric_limits<int32_t>::max())
      return fail(MBC_NO_MEMORY, "factor has more than 2^31 entries");
    p.lptr[j + 1] = (int32_t)next;
  }
  p.lind.resize(p.lptr[n]);
  for (int32_t j = 0; j < n; ++j) {
    const int32_t s = p.sup_parent[j];
    std::copy(p.set_ind.begin() + off[j], p.set_ind.begin() + p.set_ptr[s + 1],
              p.lind.begin() + p.lptr[j]);
  }
  // Theta layout (kl_chol.cu:699-706): n_s^2 per supernode
  p.th_ptr.assign(ns + 1, 0);
  p.max_set = 0;
  for (int32_t s = 0; s < ns; ++s) {
    const int64_t m = p.set_ptr[s + 1] - p.set_ptr[s];
    p.th_ptr[s + 1] = p.th_ptr[s] + m * m;
    p.max_set = std::max<int32_t>(p.max_set, (int32_t)m);
  }
  // row-wise view of L for the gather form of z = L u (columns ascending in
  // every row: the gather's summation order)
  transpose_csc(n, p.lptr, p.lind, p.rptr, p.rcol, &p.rmap, n_threads);
  p.t_super_ms = ms_since(t0);
  return MBC_OK;
}

}  // namespace mbc

// ---------------------------------------------------------------------------
// C ABI: plan
// ---------------------------------------------------------------------------
using mbc::fail;

extern "C" void mbc_plan_default_options(mbc_plan_options *opt)
{
  if (!opt) return;
  opt->rho = 3.0;
  opt->lambda = 1.5;
  opt->max_super = 2048;
  opt->n_threads = 0;
}

extern "C" mbc_status mbc_plan_create(int32_t n, const double *pts_host,
                                      const mbc_plan_options *opt, mbc_plan **out)
{
  if (!out) return fail(MBC_BAD_ARG, "out is NULL");
  *out = nullptr;
  if (n <= 0 || !pts_host) return fail(MBC_BAD_ARG, "need n > 0 points");
  mbc_plan_options o;
  mbc_plan_default_options(&o);
  if (opt) o = *opt;
  if (!(o.rho > 0) || !(o.lambda > 0) || o.max_super < 1)
    return fail(MBC_BAD_ARG, "rho and lambda must be positive and max_super >= 1");
  for (int64_t k = 0; k < 3LL * n; ++k)
    if (!std::isfinite(pts_host[k])) return fail(MBC_BAD_ARG, "points must be finite");
  mbc_plan *pl = new (std::nothrow) mbc_plan();
  if (!pl) return fail(MBC_NO_MEMORY, "plan allocation failed");
  try {
    mbc::Plan &p = pl->p;
    p.n = n;
    p.rho = (double)(float)o.rho;
    p.lambda = o.lambda;
    p.max_super = o.max_super;
    p.pts.assign(pts_host, pts_host + 3 * (size_t)n);
    mbc_status s = mbc::build_order(p, o.n_threads);
    if (s == MBC_OK) s = mbc::build_pattern(p, o.n_threads);
    if (s == MBC_OK) s = mbc::build_supernodes(p, o.n_threads);
    if (s != MBC_OK) {
      delete pl;
      return s;
    }
  } catch (const std::bad_alloc &) {
    delete pl;
    return fail(MBC_NO_MEMORY, "host allocation failed while building the plan");
  }
  *out = pl;
  return MBC_OK;
}

extern "C" mbc_status mbc_plan_destroy(mbc_plan *plan)
{
  delete plan;
  return MBC_OK;
}

extern "C" mbc_status mbc_plan_get_info(const mbc_plan *plan, mbc_plan_info *info)
{
  if (!plan || !info) return fail(MBC_BAD_ARG, "NULL argument");
  const mbc::Plan &p = plan->p;
  info->n = p.n;
  info->n_super = p.n_super;
  info->pattern_nnz = p.ptr.empty() ? 0 : p.ptr.back();
  info->factor_nnz = p.lptr.empty() ? 0 : p.lptr.back();
  info->theta_nnz = p.th_ptr.empty() ? 0 : p.th_ptr.back();
  info->max_set = p.max_set;
  info->root = p.root;
  info->t_order_ms = p.t_order_ms;
  info->t_pattern_ms = p.t_pattern_ms;
  info->t_super_ms = p.t_super_ms;
  return MBC_OK;
}

extern "C" mbc_status mbc_plan_get_order(const mbc_plan *plan, int32_t *P_host, double *scale_host)
{
  if (!plan) return fail(MBC_BAD_ARG, "NULL plan");
  const mbc::Plan &p = plan->p;
  if (P_host) std::memcpy(P_host, p.P.data(), sizeof(int32_t) * p.n);
  if (scale_host) std::memcpy(scale_host, p.scale.data(), sizeof(double) * p.n);
  return MBC_OK;
}

extern "C" mbc_status mbc_plan_get_pattern(const mbc_plan *plan, int32_t *ptr_host, int32_t *ind_host)
{
  if (!plan) return fail(MBC_BAD_ARG, "NULL plan");
  const mbc::Plan &p = plan->p;
  if (ptr_host) std::memcpy(ptr_host, p.ptr.data(), sizeof(int32_t) * p.ptr.size());
  if (ind_host) std::memcpy(ind_host, p.ind.data(), sizeof(int32_t) * p.ind.size());
  return MBC_OK;
}

extern "C" mbc_status mbc_plan_get_supernodes(const mbc_plan *plan, int32_t *sup_ptr_host,
                                              int32_t *sup_ind_host, int32_t *sup_parent_host)
{
  if (!plan) return fail(MBC_BAD_ARG, "NULL plan");
  const mbc::Plan &p = plan->p;
  if (sup_ptr_host) std::memcpy(sup_ptr_host, p.sup_ptr.data(), sizeof(int32_t) * p.sup_ptr.size());
  if (sup_ind_host) std::memcpy(sup_ind_host, p.sup_ind.data(), sizeof(int32_t) * p.sup_ind.size());
  if (sup_parent_host)
    std::memcpy(sup_parent_host, p.sup_parent.data(), sizeof(int32_t) * p.sup_parent.size());
  return MBC_OK;
}

extern "C" mbc_status mbc_plan_get_factor_pattern(const mbc_plan *plan, int32_t *lptr_host,
                                                  int32_t *lind_host)
{
  if (!plan) return fail(MBC_BAD_ARG, "NULL plan");
  const mbc::Plan &p = plan->p;
  if (lptr_host) std::memcpy(lptr_host, p.lptr.data(), sizeof(int32_t) * p.lptr.size());
  if (lind_host) std::memcpy(lind_host, p.lind.data(), sizeof(int32_t) * p.lind.size());
  return MBC_OK;
}

extern "C" mbc_status mbc_plan_get_factor_rows(const mbc_plan *plan, int32_t *rptr_host, int32_t *rcol_host,
                                               int32_t *rmap_host)
{
  if (!plan) return fail(MBC_BAD_ARG, "NULL plan");
  const mbc::Plan &p = plan->p;
  if (rptr_host) std::memcpy(rptr_host, p.rptr.data(), sizeof(int32_t) * p.rptr.size());
  if (rcol_host) std::memcpy(rcol_host, p.rcol.data(), sizeof(int32_t) * p.rcol.size());
  if (rmap_host) std::memcpy(rmap_host, p.rmap.data(), sizeof(int32_t) * p.rmap.size());
  return MBC_OK;
}
