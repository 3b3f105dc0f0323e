/*
 * mbc_oracle.c -- CPU ORACLE for the MFS solve path.  TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C and FP64, the reference algorithm of
 * fastMBCUI's MFS solve path so that the CUDA product can be checked against
 * it.  Only tests/, the smoke check and the CPU-baseline leg of bench.py may
 * load it.  The product library never links or calls it.
 *
 * Parity pin: the maximin ordering and the kd-tree radius search are checked
 * against the reference's own maxmin.h / nanoflann.hpp, compiled by
 * oracle/Makefile into oracle/_ref (see oracle/ref_driver.cpp).  The pattern,
 * aggregation and supernodal pattern are restated from preprocess.h, whose
 * Eigen dependency cannot be built here; the factor and PCG are restated from
 * kl_chol.cu.  Each function names the reference lines it follows.
 *
 * Arithmetic conventions that must match the reference bit for bit:
 *   squared distance  = (dx*dx + dy*dy) + dz*dz, each product rounded, no FMA
 *   (maxmin.h:370-374, Eigen squaredNorm over a 3-vector, nanoflann
 *   L2_Adaptor::evalMetric).  Build with -ffp-contract=off.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OK 0
#define ORC_ERR_ARG 1
#define ORC_ERR_NOMEM 2
#define ORC_ERR_COVERAGE 3

static double sq3(const double *a, const double *b)
{
  const double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
  return (dx * dx + dy * dy) + dz * dz;
}

/* ------------------------------------------------------------------------ */
/* Maximin ordering: restates maxmin.h:184-293 (heap), :295-336 (ijlookup),  */
/* :440-464 (determineChildren_3d), :588-665 (create_ordering_3d) and        */
/* preprocess.h:782-831 (root choice, reversal).  No boundary: dist_bd=1e16. */
/* ------------------------------------------------------------------------ */

typedef struct {
  int n;
  double *dist;   /* heap slot -> key */
  int32_t *id;    /* heap slot -> point id */
  int32_t *slot;  /* point id -> heap slot */
} orc_heap;

/* maxmin.h:194-263: one sift-down step; returns the child slot moved to or -1 */
static int heap_step(orc_heap *h, int a)
{
  const int l = 2 * a + 1, r = 2 * a + 2;
  int c;
  if (l >= h->n) return -1;
  if (r >= h->n) {
    if (!(h->dist[a] < h->dist[l])) return -1;
    c = l;
  } else if (h->dist[l] > h->dist[r]) {
    if (!(h->dist[a] < h->dist[l])) return -1;
    c = l;
  } else {
    if (!(h->dist[a] < h->dist[r])) return -1;
    c = r;
  }
  {
    const double td = h->dist[a];
    const int32_t ti = h->id[a];
    h->dist[a] = h->dist[c];
    h->dist[c] = td;
    h->id[a] = h->id[c];
    h->id[c] = ti;
    h->slot[h->id[a]] = a;
    h->slot[h->id[c]] = c;
  }
  return c;
}

/* maxmin.h:266-271: set a key and sift down only */
static void heap_update(orc_heap *h, int a, double d)
{
  h->dist[a] = d;
  while (a >= 0) a = heap_step(h, a);
}

/* Root choice of preprocess.h:786-814: first point strictly closest to the
 * column-wise minimum corner, starting from 1e10. */
int orc_root(int n, const double *pts)
{
  double corner[3];
  int k, best = -1;
  double bd = 1e10;
  if (n <= 0) return -1;
  corner[0] = pts[0];
  corner[1] = pts[1];
  corner[2] = pts[2];
  for (k = 1; k < n; ++k) {
    int d;
    for (d = 0; d < 3; ++d)
      if (pts[3 * k + d] < corner[d]) corner[d] = pts[3 * k + d];
  }
  for (k = 0; k < n; ++k) {
    const double d = sq3(&pts[3 * k], corner);
    if (d < bd) {
      bd = d;
      best = k;
    }
  }
  return best;
}

/*
 * Ordering.  Outputs seq[k] = point chosen at step k (coarse to fine),
 * dists[k] = its length scale.  Returns ORC_OK.
 */
int orc_maximin_seq(int n, const double *pts, int root, int32_t *seq, double *dists)
{
  orc_heap h;
  int32_t *li = NULL, *lj = NULL, *parents = NULL;
  int64_t lcap, lsize = 0;
  int pres = 0, k;
  if (n <= 0 || root < 0 || root >= n) return ORC_ERR_ARG;
  h.n = n;
  h.dist = (double *)malloc(sizeof(double) * n);
  h.id = (int32_t *)malloc(sizeof(int32_t) * n);
  h.slot = (int32_t *)malloc(sizeof(int32_t) * n);
  li = (int32_t *)malloc(sizeof(int32_t) * (n + 1));
  lcap = n;
  lj = (int32_t *)malloc(sizeof(int32_t) * lcap);
  parents = (int32_t *)malloc(sizeof(int32_t) * n);
  if (!h.dist || !h.id || !h.slot || !li || !lj || !parents) {
    free(h.dist); free(h.id); free(h.slot); free(li); free(lj); free(parents);
    return ORC_ERR_NOMEM;
  }
  /* heapInit, maxmin.h:274-293: full internal nodes 10000, others +inf */
  for (k = 0; k < n; ++k) {
    h.dist[k] = (2 * k + 2 < n) ? 10000.0 : INFINITY;
    h.id[k] = k;
    h.slot[k] = k;
  }
  li[0] = 0;
  li[1] = 0;
  /* first parent: every point is a child of the root (maxmin.h:637-646) */
  seq[0] = root;
  dists[0] = 0.0;
  for (k = 0; k < n; ++k) {
    const double d2 = sq3(&pts[3 * root], &pts[3 * k]);
    const double d = sqrt(d2);
    lj[lsize++] = k;
    li[1] = (int32_t)lsize;
    if (d > dists[0]) dists[0] = d;
    heap_update(&h, h.slot[k], d < 1e16 ? d : 1e16);
    parents[k] = 0;
  }
  /* main loop, maxmin.h:651-657 with determineChildren_3d, :440-464 */
  for (k = 1; k < n; ++k) {
    const int32_t piv = h.id[0];
    const double pd = h.dist[0];
    int64_t kk, kmin, kmax;
    seq[k] = piv;
    dists[k] = pd;
    kmin = li[parents[piv]];
    kmax = li[parents[piv] + 1];
    ++pres;
    li[pres + 1] = li[pres];
    for (kk = kmin; kk < kmax; ++kk) {
      const int32_t j = lj[kk];
      const double t2 = sq3(&pts[3 * piv], &pts[3 * j]);
      if (t2 < pd * pd) {
        double jd = h.dist[h.slot[j]];
        if (t2 < jd * jd) {
          const double s = sqrt(t2);
          const double nd = s < 1e16 ? s : 1e16;
          heap_update(&h, h.slot[j], nd);
          jd = nd;
        }
        if (lsize == lcap) {
          int32_t *nl;
          lcap *= 2;
          nl = (int32_t *)realloc(lj, sizeof(int32_t) * lcap);
          if (!nl) {
            free(h.dist); free(h.id); free(h.slot); free(li); free(lj); free(parents);
            return ORC_ERR_NOMEM;
          }
          lj = nl;
        }
        lj[lsize++] = j;
        ++li[pres + 1];
        if (sqrt(t2) + jd < pd) parents[j] = k;
      }
    }
  }
  free(h.dist); free(h.id); free(h.slot); free(li); free(lj); free(parents);
  return ORC_OK;
}

/*
 * fast_fps (preprocess.h:782-831): P[seq[i]] = n-1-i, scale = reversed dists.
 * P maps an original index to its position in the fine-to-coarse ordering.
 */
int orc_order(int n, const double *pts, int32_t *P, double *scale)
{
  int32_t *seq;
  double *d;
  int i, rc, root;
  if (n <= 0) return ORC_ERR_ARG;
  root = orc_root(n, pts);
  if (root < 0) return ORC_ERR_ARG;
  seq = (int32_t *)malloc(sizeof(int32_t) * n);
  d = (double *)malloc(sizeof(double) * n);
  if (!seq || !d) { free(seq); free(d); return ORC_ERR_NOMEM; }
  rc = orc_maximin_seq(n, pts, root, seq, d);
  if (rc == ORC_OK) {
    for (i = 0; i < n; ++i) P[i] = -1;
    for (i = 0; i < n; ++i) {
      if (P[seq[i]] != -1) { rc = ORC_ERR_COVERAGE; break; }
      P[seq[i]] = n - 1 - i;
      scale[n - 1 - i] = d[i];
    }
  }
  free(seq);
  free(d);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* MRA sparsity pattern, preprocess.h:235-316 with dim = 1.  Column j (new   */
/* order) lists rows i >= j with |x_I - x_J|^2 < min((rho l_i)^2,(rho l_j)^2)*/
/* sorted ascending.  Brute force over all pairs with the exact predicate.   */
/* ------------------------------------------------------------------------ */

/* ppts: points in NEW order (n x 3).  Two passes: count (ind == NULL), fill. */
int64_t orc_pattern(int n, const double *ppts, const double *scale, double rho,
                    int32_t *ptr, int32_t *ind)
{
  int64_t total = 0;
  int j;
  if (!ind) {
    int64_t *cnt = (int64_t *)calloc((size_t)n, sizeof(int64_t));
    if (!cnt) return -1;
#pragma omp parallel for schedule(dynamic, 64)
    for (j = 0; j < n; ++j) {
      const double lj = rho * scale[j];
      int64_t c = 0;
      int i;
      for (i = j; i < n; ++i) {
        const double li = rho * scale[i];
        const double a = li * li, b = lj * lj;
        if (sq3(&ppts[3 * i], &ppts[3 * j]) < (a < b ? a : b)) ++c;
      }
      cnt[j] = c;
    }
    ptr[0] = 0;
    for (j = 0; j < n; ++j) {
      total += cnt[j];
      ptr[j + 1] = (int32_t)total;
    }
    free(cnt);
    return total;
  }
#pragma omp parallel for schedule(dynamic, 64)
  for (j = 0; j < n; ++j) {
    const double lj = rho * scale[j];
    int32_t c = ptr[j];
    int i;
    for (i = j; i < n; ++i) {
      const double li = rho * scale[i];
      const double a = li * li, b = lj * lj;
      if (sq3(&ppts[3 * i], &ppts[3 * j]) < (a < b ? a : b)) ind[c++] = i;
    }
  }
  return ptr[n];
}

/* ------------------------------------------------------------------------ */
/* Greedy supernodes, preprocess.h:541-602 (dim 1, one group {0,n}).         */
/* ------------------------------------------------------------------------ */
int orc_aggregate(int n, const int32_t *ptr, const int32_t *ind, const double *scale,
                  double lambda, int max_super, int32_t *sup_ptr, int32_t *sup_ind,
                  int32_t *sup_parent, int32_t *n_super)
{
  unsigned char *vis = (unsigned char *)calloc((size_t)n, 1);
  int j, ns = 0, pos = 0;
  if (!vis) return ORC_ERR_NOMEM;
  sup_ptr[0] = 0;
  for (j = 0; j < n; ++j) {
    int32_t k, size = 0;
    if (vis[j]) continue;
    for (k = ptr[j]; k < ptr[j + 1]; ++k) {
      const int32_t i = ind[k];
      if (!vis[i] && scale[i] <= lambda * scale[j]) {
        vis[i] = 1;
        sup_ind[pos++] = i;
        sup_parent[i] = ns;
        ++size;
        if (size >= max_super) break;
      }
    }
    ++ns;
    sup_ptr[ns] = pos;
  }
  free(vis);
  *n_super = ns;
  /* preprocess.h:593: every point must be covered */
  return pos == n ? ORC_OK : ORC_ERR_COVERAGE;
}

/* ------------------------------------------------------------------------ */
/* Supernodal pattern, preprocess.h:604-671: each supernode's row set is the */
/* sorted union of the rows of its columns; column j keeps the suffix >= j.  */
/* Outputs set_ptr/set_ind (per supernode row set) and lptr/lind (per col).  */
/* ------------------------------------------------------------------------ */
int64_t orc_super_sets(int n, const int32_t *ptr, const int32_t *ind, int n_super,
                       const int32_t *sup_parent, int32_t *set_ptr, int32_t *set_ind)
{
  /* PT column i lists columns J with (i, J) in the pattern, ascending J; the
   * reference appends i to idx_set[parent(J)] for i ascending, then uniques. */
  int32_t *last = (int32_t *)malloc(sizeof(int32_t) * (size_t)n_super);
  int32_t *tptr = (int32_t *)calloc((size_t)n + 1, sizeof(int32_t));
  int32_t *tind = NULL, *fill = NULL;
  int64_t nnz = ptr[n], total = 0;
  int i, j, s;
  if (!last || !tptr) { free(last); free(tptr); return -1; }
  for (j = 0; j < n; ++j)
    for (int32_t k = ptr[j]; k < ptr[j + 1]; ++k) ++tptr[ind[k] + 1];
  for (i = 0; i < n; ++i) tptr[i + 1] += tptr[i];
  tind = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nnz > 0 ? nnz : 1));
  fill = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
  if (!tind || !fill) { free(last); free(tptr); free(tind); free(fill); return -1; }
  memcpy(fill, tptr, sizeof(int32_t) * n);
  for (j = 0; j < n; ++j)
    for (int32_t k = ptr[j]; k < ptr[j + 1]; ++k) tind[fill[ind[k]]++] = j;
  /* count */
  for (s = 0; s < n_super; ++s) last[s] = -1;
  if (set_ind == NULL) {
    int32_t *cnt = (int32_t *)calloc((size_t)n_super, sizeof(int32_t));
    for (i = 0; i < n; ++i)
      for (int32_t k = tptr[i]; k < tptr[i + 1]; ++k) {
        s = sup_parent[tind[k]];
        if (last[s] != i) { last[s] = i; ++cnt[s]; }
      }
    set_ptr[0] = 0;
    for (s = 0; s < n_super; ++s) { total += cnt[s]; set_ptr[s + 1] = (int32_t)total; }
    free(cnt);
  } else {
    {
      int32_t *pos = (int32_t *)malloc(sizeof(int32_t) * (size_t)n_super);
      for (s = 0; s < n_super; ++s) pos[s] = set_ptr[s];
      for (i = 0; i < n; ++i)
        for (int32_t k = tptr[i]; k < tptr[i + 1]; ++k) {
          s = sup_parent[tind[k]];
          if (last[s] != i) { last[s] = i; set_ind[pos[s]++] = i; }
        }
      free(pos);
    }
    total = set_ptr[n_super];
  }
  free(last); free(tptr); free(tind); free(fill);
  return total;
}

static int32_t lower_bound_i32(const int32_t *a, int32_t lo, int32_t hi, int32_t v)
{
  while (lo < hi) {
    const int32_t mid = lo + (hi - lo) / 2;
    if (a[mid] < v) lo = mid + 1; else hi = mid;
  }
  return lo;
}

/* Column pattern of the factor: suffix of the owning supernode's row set. */
int64_t orc_super_pattern(int n, const int32_t *sup_parent, const int32_t *set_ptr,
                          const int32_t *set_ind, int32_t *lptr, int32_t *lind)
{
  int j;
  if (!lind) {
    int64_t t = 0;
    lptr[0] = 0;
    for (j = 0; j < n; ++j) {
      const int32_t s = sup_parent[j];
      const int32_t b = lower_bound_i32(set_ind, set_ptr[s], set_ptr[s + 1], j);
      t += set_ptr[s + 1] - b;
      lptr[j + 1] = (int32_t)t;
    }
    return t;
  }
  for (j = 0; j < n; ++j) {
    const int32_t s = sup_parent[j];
    const int32_t b = lower_bound_i32(set_ind, set_ptr[s], set_ptr[s + 1], j);
    memcpy(&lind[lptr[j]], &set_ind[b], sizeof(int32_t) * (size_t)(set_ptr[s + 1] - b));
  }
  return lptr[n];
}

/* ------------------------------------------------------------------------ */
/* Operator K (collocation rows x source columns), FP64.                     */
/* Point kernel (kernels.h:24-40 scaled by coef):                            */
/*   K(i,j) = coef * ((x_i - y_j) . n_i) / |x_i - y_j|^3                     */
/* or a dense row-major Nf x N matrix M (the mfs_torch op's input).          */
/* Columns are addressed in the ORIGINAL source order.                       */
/* ------------------------------------------------------------------------ */
typedef struct {
  int nf, n;
  const double *M;   /* dense row-major nf x n, or NULL */
  const double *x;   /* nf x 3 collocation points */
  const double *nx;  /* nf x 3 normals */
  const double *y;   /* n x 3 sources */
  double coef;
} orc_op;

static double op_entry(const orc_op *op, int i, int j)
{
  if (op->M) return op->M[(size_t)i * op->n + j];
  {
    const double *xi = &op->x[3 * i], *ni = &op->nx[3 * i], *yj = &op->y[3 * j];
    const double r0 = xi[0] - yj[0], r1 = xi[1] - yj[1], r2 = xi[2] - yj[2];
    const double r2s = (r0 * r0 + r1 * r1) + r2 * r2;
    const double r1s = sqrt(r2s);
    const double rn = (r0 * ni[0] + r1 * ni[1]) + r2 * ni[2];
    return op->coef * rn / (r1s * r2s);
  }
}

/* w (nf x R, row-major) = K v (n x R, row-major; v in original order) */
void orc_apply_K(int nf, int n, const double *M, const double *x, const double *nx,
                 const double *y, double coef, int R, const double *v, double *w)
{
  orc_op op = {nf, n, M, x, nx, y, coef};
  int i;
#pragma omp parallel for schedule(static)
  for (i = 0; i < nf; ++i) {
    int r, j;
    for (r = 0; r < R; ++r) w[(size_t)i * R + r] = 0.0;
    for (j = 0; j < n; ++j) {
      const double k = op_entry(&op, i, j);
      for (r = 0; r < R; ++r) w[(size_t)i * R + r] += k * v[(size_t)j * R + r];
    }
  }
}

/* t (n x R) = K^T w (nf x R) */
void orc_apply_KT(int nf, int n, const double *M, const double *x, const double *nx,
                  const double *y, double coef, int R, const double *w, double *t)
{
  orc_op op = {nf, n, M, x, nx, y, coef};
  int j;
#pragma omp parallel for schedule(static)
  for (j = 0; j < n; ++j) {
    int r, i;
    for (r = 0; r < R; ++r) t[(size_t)j * R + r] = 0.0;
    for (i = 0; i < nf; ++i) {
      const double k = op_entry(&op, i, j);
      for (r = 0; r < R; ++r) t[(size_t)j * R + r] += k * w[(size_t)i * R + r];
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Supernodal KL factor, kl_chol.cu:166-223 (Theta, reversed, column-major), */
/* :16-36 (A = U^T U in place), :38-53 + :362-387 (leading-block back solve, */
/* reverse).  Theta entries are Gram entries K(:,I)^T K(:,J) (kernels.h:69-84)*/
/* th_ptr[s+1] = th_ptr[s] + n_s^2 (kl_chol.cu:699-706).                     */
/* perm_inv[p] = original index of the point at new position p.              */
/* ------------------------------------------------------------------------ */
int orc_factor(int nf, int n, const double *M, const double *x, const double *nx,
               const double *y, double coef, const int32_t *perm_inv, int n_super,
               const int32_t *sup_ptr, const int32_t *sup_ind, const int32_t *set_ptr,
               const int32_t *set_ind, const int64_t *th_ptr, double *th,
               const int32_t *lptr, const int32_t *lind, double *lval,
               int32_t *bad_pivots)
{
  orc_op op = {nf, n, M, x, nx, y, coef};
  int s;
  int bad = 0;
  (void)lind;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : bad)
  for (s = 0; s < n_super; ++s) {
    const int32_t b = set_ptr[s], ns = set_ptr[s + 1] - set_ptr[s];
    double *A = &th[th_ptr[s]];
    double *Ks = (double *)malloc(sizeof(double) * (size_t)nf * (ns > 0 ? ns : 1));
    int p, q, i, j, k;
    /* gather K(:, I_s) columns (column-major nf x ns) */
    for (p = 0; p < ns; ++p) {
      const int col = perm_inv[set_ind[b + p]];
      for (i = 0; i < nf; ++i) Ks[(size_t)p * nf + i] = op_entry(&op, i, col);
    }
    /* Theta_rev[rev_p + rev_q*ns] = K(:,I_p)^T K(:,I_q) */
    for (p = 0; p < ns; ++p)
      for (q = p; q < ns; ++q) {
        double g = 0.0;
        for (i = 0; i < nf; ++i) g += Ks[(size_t)p * nf + i] * Ks[(size_t)q * nf + i];
        A[(ns - 1 - p) + (size_t)(ns - 1 - q) * ns] = g;
        A[(ns - 1 - q) + (size_t)(ns - 1 - p) * ns] = g;
      }
    free(Ks);
    /* dense_chol_fac: A = U^T U, U in the upper triangle */
    for (j = 0; j < ns; ++j) {
      double dot;
      for (i = 0; i < j; ++i) {
        dot = 0.0;
        for (k = 0; k < i; ++k) dot += A[k + (size_t)j * ns] * A[k + (size_t)i * ns];
        A[i + (size_t)j * ns] = (A[i + (size_t)j * ns] - dot) / A[i + (size_t)i * ns];
      }
      dot = 0.0;
      for (k = 0; k < j; ++k) dot += A[k + (size_t)j * ns] * A[k + (size_t)j * ns];
      {
        const double piv = A[j + (size_t)j * ns] - dot;
        if (!(piv > 0.0)) ++bad;
        A[j + (size_t)j * ns] = sqrt(piv);
      }
    }
    /* back solve per column of the supernode */
    for (p = sup_ptr[s]; p < sup_ptr[s + 1]; ++p) {
      const int32_t col = sup_ind[p];
      const int32_t nb = lptr[col + 1] - lptr[col];
      double *bv = &lval[lptr[col]];
      const int end = nb - 1;
      for (i = 0; i < nb; ++i) bv[i] = 0.0;
      bv[nb - 1] = 1.0;
      for (i = 0; i < nb; ++i) {
        for (j = 0; j < i; ++j) bv[end - i] -= bv[end - j] * A[(end - i) + (size_t)(end - j) * ns];
        bv[end - i] /= A[(end - i) + (size_t)(end - i) * ns];
      }
      for (i = 0; i < nb / 2; ++i) {
        const double t = bv[i];
        bv[i] = bv[nb - 1 - i];
        bv[nb - 1 - i] = t;
      }
    }
  }
  if (bad_pivots) *bad_pivots = bad;
  return ORC_OK;
}

/* z = L (L^T r), L in CSC (lptr, lind, lval) over the new order */
void orc_precond(int n, const int32_t *lptr, const int32_t *lind, const double *lval,
                 const double *r, double *tmp, double *z)
{
  int j;
#pragma omp parallel for schedule(static)
  for (j = 0; j < n; ++j) {
    double acc = 0.0;
    for (int32_t k = lptr[j]; k < lptr[j + 1]; ++k) acc += lval[k] * r[lind[k]];
    tmp[j] = acc;
  }
  for (j = 0; j < n; ++j) z[j] = 0.0;
  for (j = 0; j < n; ++j)
    for (int32_t k = lptr[j]; k < lptr[j + 1]; ++k) z[lind[k]] += lval[k] * tmp[j];
}

static double dotv(int n, const double *a, const double *b)
{
  double s = 0.0;
  int i;
  for (i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

/*
 * PCG on (K_p^T K_p) x = b, kl_chol.cu:891-1088 (forward: b = K_p^T f) and
 * :1090-1264 (adjoint: b given).  x0 = 0, stop when |r|^2 < tol^2 |b|^2 on the
 * recursive residual, early exit when |b|^2 < 1e-16.  All in the NEW order:
 * f has nf entries; b, x have n entries (b only read when adjoint != 0).
 * Returns iterations; *relres = sqrt(|r|^2/|b|^2).
 */
int orc_pcg(int nf, int n, const double *M, const double *x, const double *nx,
            const double *y, double coef, const int32_t *perm_inv, const int32_t *lptr,
            const int32_t *lind, const double *lval, int adjoint, const double *f,
            const double *bvec, int precond, int maxits, double tol, double *xout,
            double *relres)
{
  double *r = (double *)malloc(sizeof(double) * n);
  double *p = (double *)malloc(sizeof(double) * n);
  double *z = (double *)malloc(sizeof(double) * n);
  double *t = (double *)malloc(sizeof(double) * n);
  double *tmp = (double *)malloc(sizeof(double) * n);
  double *po = (double *)malloc(sizeof(double) * n);
  double *to = (double *)malloc(sizeof(double) * n);
  double *w = (double *)malloc(sizeof(double) * nf);
  double rhs2, thr, absnew, resd2 = 0.0;
  int it = 0, k;
  if (!r || !p || !z || !t || !tmp || !po || !to || !w) {
    free(r); free(p); free(z); free(t); free(tmp); free(po); free(to); free(w);
    return -1;
  }
  /* b */
  if (adjoint) {
    for (k = 0; k < n; ++k) r[k] = bvec[k];
  } else {
    orc_apply_KT(nf, n, M, x, nx, y, coef, 1, f, to);
    for (k = 0; k < n; ++k) r[k] = to[perm_inv[k]];
  }
  for (k = 0; k < n; ++k) xout[k] = 0.0;
  rhs2 = dotv(n, r, r);
  if (rhs2 < 1e-16) {
    *relres = 0.0;
    free(r); free(p); free(z); free(t); free(tmp); free(po); free(to); free(w);
    return 0;
  }
  thr = tol * tol * rhs2;
  if (precond) orc_precond(n, lptr, lind, lval, r, tmp, p);
  else memcpy(p, r, sizeof(double) * n);
  absnew = dotv(n, r, p);
  while (it < maxits) {
    double alpha, beta, absold;
    ++it;
    for (k = 0; k < n; ++k) po[perm_inv[k]] = p[k];
    orc_apply_K(nf, n, M, x, nx, y, coef, 1, po, w);
    orc_apply_KT(nf, n, M, x, nx, y, coef, 1, w, to);
    for (k = 0; k < n; ++k) t[k] = to[perm_inv[k]];
    alpha = absnew / dotv(n, p, t);
    for (k = 0; k < n; ++k) xout[k] += alpha * p[k];
    for (k = 0; k < n; ++k) r[k] -= alpha * t[k];
    resd2 = dotv(n, r, r);
    if (resd2 < thr) break;
    if (precond) orc_precond(n, lptr, lind, lval, r, tmp, z);
    else memcpy(z, r, sizeof(double) * n);
    absold = absnew;
    absnew = dotv(n, r, z);
    beta = absnew / absold;
    for (k = 0; k < n; ++k) p[k] = beta * p[k] + z[k];
  }
  *relres = sqrt(resd2 / rhs2);
  free(r); free(p); free(z); free(t); free(tmp); free(po); free(to); free(w);
  return it;
}

/*
 * orc_pcg on R forward columns at once: the same per-column recurrence
 * (kl_chol.cu:891-1088 run once per column, mfs_torch_ops.cu:162-171), with
 * the K / K^T passes shared by the columns that still iterate so that each
 * kernel entry is evaluated once per pass for all of them.  Every column's
 * arithmetic is that of orc_pcg alone: orc_apply_K / orc_apply_KT sum each
 * (row, column) over the same index order for any R, and the dot products
 * and preconditioner run on per-column vectors.  A column stops exactly
 * where orc_pcg would; its x, iterations and relres are those orc_pcg
 * returns.  F: nf x R row-major (original row order); xout: n x R row-major
 * in the NEW order; iters[R], relres[R].  Returns 0, or -1 on allocation
 * failure.
 */
int orc_pcg_many(int nf, int n, const double *M, const double *x, const double *nx,
                 const double *y, double coef, const int32_t *perm_inv, const int32_t *lptr,
                 const int32_t *lind, const double *lval, int R, const double *F, int maxits,
                 double tol, double *xout, int32_t *iters, double *relres)
{
  const size_t nn = (size_t)n, nR = (size_t)n * R;
  double *r = (double *)malloc(sizeof(double) * nR);   /* per column, contiguous */
  double *p = (double *)malloc(sizeof(double) * nR);
  double *z = (double *)malloc(sizeof(double) * nR);
  double *xc = (double *)malloc(sizeof(double) * nR);
  double *tmp = (double *)malloc(sizeof(double) * nn);
  double *po = (double *)malloc(sizeof(double) * nR);  /* n x A row-major, original order */
  double *to = (double *)malloc(sizeof(double) * nR);
  double *w = (double *)malloc(sizeof(double) * (size_t)nf * R);
  double *col = (double *)malloc(sizeof(double) * nn);     /* t of one column */
  double *thr = (double *)malloc(sizeof(double) * R), *rhs2 = (double *)malloc(sizeof(double) * R);
  double *absnew = (double *)malloc(sizeof(double) * R), *resd2 = (double *)malloc(sizeof(double) * R);
  int *act = (int *)malloc(sizeof(int) * R);
  int c, k, A, i;
  if (!r || !p || !z || !xc || !tmp || !po || !to || !w || !col || !thr || !rhs2 || !absnew || !resd2 || !act) {
    free(r); free(p); free(z); free(xc); free(tmp); free(po); free(to); free(w); free(col);
    free(thr); free(rhs2); free(absnew); free(resd2); free(act);
    return -1;
  }
  /* b = K_p^T f per column (one R-column pass: same sums as R = 1) */
  orc_apply_KT(nf, n, M, x, nx, y, coef, R, F, to);
  A = 0;
  for (c = 0; c < R; ++c) {
    double *rc = r + (size_t)c * nn;
    for (k = 0; k < n; ++k) rc[k] = to[(size_t)perm_inv[k] * R + c];
    for (k = 0; k < n; ++k) xc[(size_t)c * nn + k] = 0.0;
    rhs2[c] = dotv(n, rc, rc);
    iters[c] = 0;
    resd2[c] = 0.0;
    relres[c] = 0.0;
    if (rhs2[c] < 1e-16) continue;
    thr[c] = tol * tol * rhs2[c];
    orc_precond(n, lptr, lind, lval, rc, tmp, p + (size_t)c * nn);
    absnew[c] = dotv(n, rc, p + (size_t)c * nn);
    act[A++] = c;
  }
  while (A > 0) {
    int A2 = 0;
    for (i = 0; i < A; ++i) {
      const double *pc = p + (size_t)act[i] * nn;
      for (k = 0; k < n; ++k) po[(size_t)perm_inv[k] * A + i] = pc[k];
    }
    orc_apply_K(nf, n, M, x, nx, y, coef, A, po, w);
    orc_apply_KT(nf, n, M, x, nx, y, coef, A, w, to);
    for (i = 0; i < A; ++i) {
      c = act[i];
      double *rc = r + (size_t)c * nn, *pc = p + (size_t)c * nn, *zc = z + (size_t)c * nn;
      double *xcc = xc + (size_t)c * nn, *t = col;
      double alpha, beta, absold;
      ++iters[c];
      for (k = 0; k < n; ++k) t[k] = to[(size_t)perm_inv[k] * A + i];
      alpha = absnew[c] / dotv(n, pc, t);
      for (k = 0; k < n; ++k) xcc[k] += alpha * pc[k];
      for (k = 0; k < n; ++k) rc[k] -= alpha * t[k];
      resd2[c] = dotv(n, rc, rc);
      if (resd2[c] < thr[c] || iters[c] >= maxits) continue;
      orc_precond(n, lptr, lind, lval, rc, tmp, zc);
      absold = absnew[c];
      absnew[c] = dotv(n, rc, zc);
      beta = absnew[c] / absold;
      for (k = 0; k < n; ++k) pc[k] = beta * pc[k] + zc[k];
      act[A2++] = c;
    }
    A = A2;
  }
  for (c = 0; c < R; ++c) {
    if (rhs2[c] >= 1e-16) relres[c] = sqrt(resd2[c] / rhs2[c]);
    for (k = 0; k < n; ++k) xout[(size_t)k * R + c] = xc[(size_t)c * nn + k];
  }
  free(r); free(p); free(z); free(xc); free(tmp); free(po); free(to); free(w); free(col);
  free(thr); free(rhs2); free(absnew); free(resd2); free(act);
  return 0;
}

/*
 * Added-mass tensor of a solved scene (the parity observable downstream of
 * the solve): core/KTAB_Mfs_spclf1d.py:123-128 with utils/torch_utils.py
 * compute_single_layer (:254-276) and compute_quadrature (:336-347).
 *   phi = SL X,  SL(i, j) = 1 / (4 pi |x_i - y_j|)
 *   Mf[6a + m, c] = -rho_f sum_{k in body a} w_k N_m(k) phi(k, c),
 *   N(k) = (n_k, (x_k - centre_a) x n_k).
 * The reference pairs its solid-angle operator with SL = 1/|x - y|; with the
 * normal-derivative operator of G = 1/(4 pi r) used here the same potential
 * carries the 1/(4 pi).  X: n x R row-major (original source order); w: nf
 * quadrature weights; body_ptr: rows of body a are [body_ptr[a], body_ptr[a+1]).
 */
void orc_added_mass(int nf, int n, const double *x, const double *nx, const double *y, int R,
                    const double *X, const double *w, int nb, const int32_t *body_ptr,
                    const double *centers, double rho_f, double *Mf)
{
  double *phi = (double *)malloc(sizeof(double) * (size_t)nf * R);
  int i;
#pragma omp parallel for schedule(static)
  for (i = 0; i < nf; ++i) {
    double *pr = phi + (size_t)i * R;
    int j, c;
    for (c = 0; c < R; ++c) pr[c] = 0.0;
    for (j = 0; j < n; ++j) {
      const double g = 1.0 / (4.0 * 3.14159265358979323846 * sqrt(sq3(&x[3 * i], &y[3 * j])));
      const double *xr = X + (size_t)j * R;
      for (c = 0; c < R; ++c) pr[c] += g * xr[c];
    }
  }
  int a;
  for (a = 0; a < nb; ++a) {
    int m, c, k;
    for (m = 0; m < 6; ++m)
      for (c = 0; c < R; ++c) Mf[(size_t)(6 * a + m) * R + c] = 0.0;
    for (k = body_ptr[a]; k < body_ptr[a + 1]; ++k) {
      const double *nk = &nx[3 * k];
      const double r0 = x[3 * k] - centers[3 * a], r1 = x[3 * k + 1] - centers[3 * a + 1],
                   r2 = x[3 * k + 2] - centers[3 * a + 2];
      const double N[6] = {nk[0], nk[1], nk[2], r1 * nk[2] - r2 * nk[1], r2 * nk[0] - r0 * nk[2],
                           r0 * nk[1] - r1 * nk[0]};
      for (m = 0; m < 6; ++m)
        for (c = 0; c < R; ++c) Mf[(size_t)(6 * a + m) * R + c] += w[k] * N[m] * phi[(size_t)k * R + c];
    }
    for (m = 0; m < 6; ++m)
      for (c = 0; c < R; ++c) Mf[(size_t)(6 * a + m) * R + c] *= -rho_f;
  }
  free(phi);
}

/*
 * Mesh collocation operator: the solid angle of face f seen from source j
 * (utils/torch_utils.py:306-334, compute_solid_angle; van Oosterom and
 * Strackee), Rk = V[F[f, k]] - S[j]:
 *   M[f, j] = 2 atan2(R1 . (R2 x R3), l1 l2 l3 + (R1.R2) l3 + (R1.R3) l2 + (R2.R3) l1).
 * Rows: every face (bodies concatenated, core/KTAB_Mfs_spclf1d.py:112);
 * columns: every source.  M is row-major n_faces x n_src.
 */
void orc_mesh_solid_angle(int n_faces, const double *V, const int32_t *F, int n_src, const double *S,
                          double *M)
{
  int f;
#pragma omp parallel for schedule(static)
  for (f = 0; f < n_faces; ++f) {
    const double *v1 = &V[3 * F[3 * f]], *v2 = &V[3 * F[3 * f + 1]], *v3 = &V[3 * F[3 * f + 2]];
    int j;
    for (j = 0; j < n_src; ++j) {
      const double *s = &S[3 * j];
      const double a[3] = {v1[0] - s[0], v1[1] - s[1], v1[2] - s[2]};
      const double b[3] = {v2[0] - s[0], v2[1] - s[1], v2[2] - s[2]};
      const double c[3] = {v3[0] - s[0], v3[1] - s[1], v3[2] - s[2]};
      const double bxc[3] = {b[1] * c[2] - b[2] * c[1], b[2] * c[0] - b[0] * c[2], b[0] * c[1] - b[1] * c[0]};
      const double num = a[0] * bxc[0] + a[1] * bxc[1] + a[2] * bxc[2];
      const double la = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
      const double lb = sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
      const double lc = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
      const double ab = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
      const double ac = a[0] * c[0] + a[1] * c[1] + a[2] * c[2];
      const double bc = b[0] * c[0] + b[1] * c[1] + b[2] * c[2];
      const double den = la * lb * lc + ab * lc + ac * lb + bc * la;
      M[(size_t)f * n_src + j] = 2.0 * atan2(num, den);
    }
  }
}

/*
 * Rigid-mode right-hand side of the mesh operator: FL @ IQ of
 * core/KTAB_Mfs_spclf1d.py:101-108 with compute_FL_matrix
 * (utils/torch_utils.py:62-75) and compute_face_centers (:49-60).  Face f of
 * body b has the area-weighted normal s = (v2 - v1) x (v3 - v1) / 2 and the
 * lever arm r = (v1 + v2 + v3) / 3 - y_b; FL's row (r x s, s) times
 * IQ = [[0, I], [I, 0]] puts (s, r x s) in columns 6b .. 6b + 5.
 * Out: row-major n_faces x 6 n_bodies, zero outside the face's body block.
 */
void orc_mesh_rhs(int n_faces, const double *V, const int32_t *F, const int32_t *face_body, int n_bodies,
                  const double *body_pos, double *out)
{
  int f;
  memset(out, 0, sizeof(double) * (size_t)n_faces * 6 * n_bodies);
  for (f = 0; f < n_faces; ++f) {
    const double *v1 = &V[3 * F[3 * f]], *v2 = &V[3 * F[3 * f + 1]], *v3 = &V[3 * F[3 * f + 2]];
    const int b = face_body[f];
    const double e1[3] = {v2[0] - v1[0], v2[1] - v1[1], v2[2] - v1[2]};
    const double e2[3] = {v3[0] - v1[0], v3[1] - v1[1], v3[2] - v1[2]};
    const double sv[3] = {(e1[1] * e2[2] - e1[2] * e2[1]) / 2.0, (e1[2] * e2[0] - e1[0] * e2[2]) / 2.0,
                          (e1[0] * e2[1] - e1[1] * e2[0]) / 2.0};
    const double r[3] = {(v1[0] + v2[0] + v3[0]) / 3.0 - body_pos[3 * b],
                         (v1[1] + v2[1] + v3[1]) / 3.0 - body_pos[3 * b + 1],
                         (v1[2] + v2[2] + v3[2]) / 3.0 - body_pos[3 * b + 2]};
    double *o = out + (size_t)f * 6 * n_bodies + 6 * b;
    o[0] = sv[0];
    o[1] = sv[1];
    o[2] = sv[2];
    o[3] = r[1] * sv[2] - r[2] * sv[1];
    o[4] = r[2] * sv[0] - r[0] * sv[2];
    o[5] = r[0] * sv[1] - r[1] * sv[0];
  }
}

/* ---- INT8 digit-sliced FP64 matvec ----------------------------------------
 * Restatement of the library's FP64-accurate INT8 tensor-core matvec (its own
 * design, not a reference algorithm), so that the device result can be
 * checked operation for operation:
 *   out[i, r] = coef * sum_j G[i, j] V[j, r]
 * over K cut into 2048-wide chunks; per chunk a power-of-two scale 2^a per
 * row of G (largest finite |G|; non-finite G counts as 0) and 2^b per column
 * of V (a column chunk holding a non-finite value gets b = 4096, an infinite
 * weight); T = rint(v 2^-a 2^38) as five balanced base-256 digits (the bytes
 * of (T + B) xor B, B = 0x8080808080); digit-pair levels l = p + q <= 4
 * summed exactly; comb = Horner in base 256 over the levels; sum =
 * fma((double)comb, 2^(a + b - 44), sum) chunk by chunk; out = coef * sum.
 * Returns 0, or 1 if a level sum left the INT32 range (the device
 * accumulators would have wrapped). */
#define OZ_DIGITS 5
#define OZ_W 38
#define OZ_CHUNK 2048
#define OZ_SHIFT 44
#define OZ_NONFINITE 4096

static double oz_pow2(int e)
{
  if (e < -1022) return 0.0;
  if (e > 1023) return INFINITY;
  const uint64_t b = (uint64_t)(e + 1023) << 52;
  double d;
  memcpy(&d, &b, sizeof d);
  return d;
}

static int oz_ceil_exp2(double m)
{
  uint64_t b;
  memcpy(&b, &m, sizeof b);
  const int E = (int)((b >> 52) & 0x7FF);
  if (E == 0) return b == 0 ? 0 : -1022;
  return E - 1023 + ((b & 0xFFFFFFFFFFFFFull) != 0 ? 1 : 0);
}

static void oz_digits(double v, int a, int8_t *d)
{
  const long long T = llrint((v * oz_pow2(-a)) * oz_pow2(OZ_W));
  const uint64_t tb = ((uint64_t)T + 0x8080808080ull) ^ 0x8080808080ull;
  for (int p = 0; p < OZ_DIGITS; ++p) d[p] = (int8_t)(uint8_t)((tb >> (8 * (OZ_DIGITS - 1 - p))) & 0xFF);
}

int orc_oz_apply(int M, int K, int R, const double *G, const double *V, double coef, double *out)
{
  const int nch = (K + OZ_CHUNK - 1) / OZ_CHUNK;
  double *sum = (double *)calloc((size_t)M * R + 1, sizeof(double));
  int8_t *dg = (int8_t *)malloc((size_t)M * OZ_CHUNK * OZ_DIGITS + 1);
  int8_t *dv = (int8_t *)malloc((size_t)R * OZ_CHUNK * OZ_DIGITS + 1);
  int *ea = (int *)malloc(sizeof(int) * ((size_t)M + 1));
  int *eb = (int *)malloc(sizeof(int) * ((size_t)R + 1));
  int bad = 0;
  for (int c = 0; c < nch; ++c) {
    const int k0 = c * OZ_CHUNK;
    const int kc = K - k0 < OZ_CHUNK ? K - k0 : OZ_CHUNK;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < M; ++i) {
      double m = 0.0;
      for (int j = 0; j < kc; ++j) {
        const double g = G[(size_t)i * K + k0 + j];
        if (isfinite(g)) m = fmax(m, fabs(g));
      }
      ea[i] = oz_ceil_exp2(m);
      for (int j = 0; j < kc; ++j) {
        const double g = G[(size_t)i * K + k0 + j];
        int8_t *d = dg + ((size_t)i * OZ_CHUNK + j) * OZ_DIGITS;
        if (isfinite(g)) oz_digits(g, ea[i], d);
        else memset(d, 0, OZ_DIGITS);
      }
    }
    for (int r = 0; r < R; ++r) {
      double m = 0.0;
      int finite = 1;
      for (int j = 0; j < kc; ++j) {
        const double v = V[(size_t)(k0 + j) * R + r];
        finite = finite && isfinite(v);
        m = fmax(m, fabs(v));
      }
      eb[r] = finite && isfinite(m) ? oz_ceil_exp2(m) : OZ_NONFINITE;
      for (int j = 0; j < kc; ++j)
        oz_digits(V[(size_t)(k0 + j) * R + r], eb[r], dv + ((size_t)r * OZ_CHUNK + j) * OZ_DIGITS);
    }
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int i = 0; i < M; ++i) {
      for (int r = 0; r < R; ++r) {
        long long acc[OZ_DIGITS] = {0, 0, 0, 0, 0};
        for (int j = 0; j < kc; ++j) {
          const int8_t *a = dg + ((size_t)i * OZ_CHUNK + j) * OZ_DIGITS;
          const int8_t *b = dv + ((size_t)r * OZ_CHUNK + j) * OZ_DIGITS;
          for (int p = 0; p < OZ_DIGITS; ++p)
            for (int q = 0; p + q < OZ_DIGITS; ++q) acc[p + q] += (long long)a[p] * (long long)b[q];
        }
        long long comb = 0;
        for (int l = 0; l < OZ_DIGITS; ++l) {
          if (acc[l] > 2147483647ll || acc[l] < -2147483648ll) bad = 1;
          comb = comb * 256 + acc[l];
        }
        double *s = sum + (size_t)i * R + r;
        *s = fma((double)comb, oz_pow2(ea[i] + eb[r] - OZ_SHIFT), *s);
      }
    }
  }
  for (size_t t = 0; t < (size_t)M * R; ++t) out[t] = coef * sum[t];
  free(sum);
  free(dg);
  free(dv);
  free(ea);
  free(eb);
  return bad;
}

int orc_num_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
