/*
 * mbc.h -- C ABI of the B200-native MFS solve path (libmbc.so).
 *
 * The path: maximin ordering -> KL sparsity pattern -> supernodes (host C++,
 * bit-exact to the reference), supernodal KL-Cholesky factor of (K^T K)^-1
 * and PCG on the normal equations (CUDA, sm_100a).  K is the MFS collocation
 * operator: a caller-provided dense matrix (the mfs_torch operator's input) or
 * the Laplace point kernel evaluated on the fly.
 *
 * Conventions
 *   - Every function returns mbc_status and never exits the process.
 *     mbc_last_error() gives a message for the calling thread.
 *   - Arrays named *_host live in host memory; every other array pointer is a
 *     device pointer on the current CUDA device.
 *   - Matrices are row-major.  A "source-space" array (n x R) is indexed by the
 *     ORIGINAL source order unless its name says otherwise.
 *   - mbc_stream is cudaStream_t; NULL is the legacy default stream.
 *   - Objects are caller-owned; the library keeps no global state.
 */
#ifndef MBC_H
#define MBC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *mbc_stream;

typedef enum {
  MBC_OK = 0,
  MBC_NOT_CONVERGED = 1, /* max iterations reached above the tolerance */
  MBC_BREAKDOWN = 2,     /* PCG curvature p.Ap <= 0 or NaN */
  MBC_NONSPD_PIVOT = 3,  /* a supernode Cholesky pivot was <= 0 even after the FP64 retry */
  MBC_BAD_ARG = 4,
  MBC_CUDA_ERROR = 5,
  MBC_TIMEOUT = 6,       /* a bounded device wait gave up */
  MBC_NO_MEMORY = 7,
  MBC_COVERAGE = 8,      /* aggregation did not cover every point (e.g. duplicate points) */
  MBC_UNSUPPORTED = 9
} mbc_status;

typedef enum { MBC_F64 = 0, MBC_F32 = 1 } mbc_dtype;

const char *mbc_status_string(mbc_status s);
const char *mbc_last_error(void);
/* Library version as 10000*major + 100*minor + patch. */
int32_t mbc_version(void);

/* ------------------------------------------------------------------------ */
/* Plan: ordering, pattern, supernodes (host).                               */
/* Replaces klchol::fps_sampler (src/preprocess.h:17-671): fps_sampler(pts), */
/* compute('F'), P(), simpl_sparsity(rho, 1, PATT), aggregate(1, {0,N},      */
/* PATT, lambda, ..., max_super), super_sparsity(1, PATT, parent, SUP_PATT), */
/* as called by mfs_torch/csrc/mfs_torch_ops.cu:51-55 and :114-116.          */
/* ------------------------------------------------------------------------ */
typedef struct mbc_plan mbc_plan;

typedef struct {
  double rho;        /* pattern radius factor; used as (double)(float)rho (mfs_torch_ops.cu:114) */
  double lambda;     /* supernode scale ratio, 1.5 in the reference */
  int32_t max_super; /* max columns per supernode, 2048 in the reference */
  int32_t n_threads; /* host threads for the ordering's long scans and the pattern; 0 = all */
} mbc_plan_options;

typedef struct {
  int32_t n;
  int32_t n_super;
  int64_t pattern_nnz;
  int64_t factor_nnz;
  int64_t theta_nnz;  /* sum over supernodes of n_s^2 */
  int32_t max_set;    /* largest supernode row set */
  int32_t root;       /* original index of the first (coarsest) point */
  double t_order_ms, t_pattern_ms, t_super_ms;
} mbc_plan_info;

void mbc_plan_default_options(mbc_plan_options *opt);
/* pts_host: n x 3 (double).  The mfs_torch operator widens float32 points. */
mbc_status mbc_plan_create(int32_t n, const double *pts_host, const mbc_plan_options *opt,
                           mbc_plan **out);
mbc_status mbc_plan_destroy(mbc_plan *plan);
mbc_status mbc_plan_get_info(const mbc_plan *plan, mbc_plan_info *info);
/* P[orig] = position in the fine-to-coarse order; scale in that order. */
mbc_status mbc_plan_get_order(const mbc_plan *plan, int32_t *P_host, double *scale_host);
/* MRA pattern, CSC over the new order: ptr[n+1], ind[pattern_nnz]. */
mbc_status mbc_plan_get_pattern(const mbc_plan *plan, int32_t *ptr_host, int32_t *ind_host);
mbc_status mbc_plan_get_supernodes(const mbc_plan *plan, int32_t *sup_ptr_host,
                                   int32_t *sup_ind_host, int32_t *sup_parent_host);
/* Supernodal factor pattern, CSC: lptr[n+1], lind[factor_nnz]. */
mbc_status mbc_plan_get_factor_pattern(const mbc_plan *plan, int32_t *lptr_host,
                                       int32_t *lind_host);
/* Row-wise view of the factor pattern that the preconditioner's gather
 * z = L u walks: rptr[n+1]; row i's entries rcol (their columns, ascending)
 * and rmap (their positions in lind), factor_nnz each.  For parity tests. */
mbc_status mbc_plan_get_factor_rows(const mbc_plan *plan, int32_t *rptr_host, int32_t *rcol_host,
                                    int32_t *rmap_host);

/* Morton (Z-curve) order of n points: order_host[k] = index of the k-th point
 * along the curve (21 bits per axis over the points' bounding cube, ties by
 * index).  Coordinates at pts_host[i * stride + 0..2], stride >= 3 floats.
 * No counterpart in the reference: the INT8 FP64 matvec walks its reduction
 * axes in this order (mbc_solver_set_fp64_matvec), and tests use it to
 * restate that matvec. */
mbc_status mbc_spatial_order(int32_t n, const float *pts_host, int32_t stride, int32_t *order_host);

/* ------------------------------------------------------------------------ */
/* Operator K (nf collocation rows x n source columns).                       */
/* ------------------------------------------------------------------------ */
typedef enum { MBC_OP_DENSE = 0, MBC_OP_POINT_KERNEL = 1, MBC_OP_MESH = 2 } mbc_op_kind;

typedef struct {
  int32_t kind;
  int32_t nf, n;
  /* MBC_OP_DENSE: row-major nf x n float32, row stride ldm (>= n). */
  const float *M;
  int64_t ldm;
  /* MBC_OP_POINT_KERNEL: K(i,j) = coef ((x_i - y_j).n_i) / |x_i - y_j|^3
   * (src/kernels.h:24-40 with coef = 1).  x, nx: nf x 3; y: n x 3. */
  const float *x, *nx, *y;
  double coef;
  /* MBC_OP_MESH (matrix-free form of the mesh collocation operator,
   * utils/torch_utils.py:306-334): K(f, j) = coef * the solid angle of face f
   * (vertices V[faces[f][0..2]]) seen from source y_j, evaluated on the fly
   * (the dense matrix mbc_mesh_assemble writes, never stored).  nf = faces;
   * faces: device nf x 3 int32; V: device n_vert x 3; y: device n x 3.
   * FP64 and FP32 CUDA-core matvecs (no tensor-core or INT8 form). */
  const float *V;
  const int32_t *faces;
  int32_t n_vert;
} mbc_operator;

/* ------------------------------------------------------------------------ */
/* Solver: device factor + PCG.                                               */
/* Replaces klchol::gpu_super_klchol (src/kl_chol.h:143-336): set_kernel,    */
/* build_cov_mat_LS_float, set_supernodes, set_sppatt, compute, pcg_guesss,   */
/* pcg_VpL_guesss, get_TH_val / get_val.                                     */
/* ------------------------------------------------------------------------ */
typedef struct mbc_solver mbc_solver;

/* precision MBC_F64: the plain method, FP64 throughout.
 * precision MBC_F32: matvec, factor and preconditioner in FP32; PCG scalars,
 * dot products and the true residual in FP64 with iterative refinement. */
mbc_status mbc_solver_create(const mbc_plan *plan, const mbc_operator *op, int32_t precision,
                             mbc_stream stream, mbc_solver **out);
mbc_status mbc_solver_destroy(mbc_solver *s);
/* Assemble Theta, factor every supernode, form the KL columns (kl_chol.cu:772-812). */
mbc_status mbc_solver_factor(mbc_solver *s, mbc_stream stream);
/* Copy the factor out for parity checks: lval[factor_nnz] (CSC of the plan),
 * theta[theta_nnz] (per supernode, reversed, column-major, U in the upper part;
 * NULL to skip).  Values are widened to double. */
mbc_status mbc_solver_get_factor(const mbc_solver *s, double *lval_host, double *theta_host);
/* Tile shapes of the factor kernels.  Supernodes are split by their row-set
 * size n_s into four classes: n_s <= max_ns[0] (128 threads), <= max_ns[1]
 * (256), <= max_ns[2] (512), each with Theta_s in shared memory, and larger
 * ones (512 threads, Theta_s in global memory).  tile_rows[c] is how many
 * collocation rows of the K panel a class stages per pass (class 3, and any
 * class whose shared memory would not fit, use at most that many).  The
 * shapes change the order of the Gram sums (results agree to rounding), not
 * the method.  In FP32 factors, supernodes with tc_min_ns <= n_s <= 192 form
 * Theta_s on the tensor cores (tcgen05, 3xTF32 with FP32 chunk sums) before
 * their class kernel factors it; 0 keeps every Gram on the CUDA cores.  FP64
 * factors and the FP64 retries always use the CUDA cores.  No counterpart in
 * the reference (one thread per supernode, kl_chol.cu:166-223). */
typedef struct {
  int32_t max_ns[3];    /* increasing, 1 .. 144 */
  int32_t tile_rows[4]; /* 1 .. 256 */
  int32_t tc_min_ns;    /* 0, or 32 .. 192 (default 64) */
} mbc_factor_tiles;

void mbc_factor_default_tiles(mbc_factor_tiles *tiles);
mbc_status mbc_solver_set_factor_tiles(mbc_solver *s, const mbc_factor_tiles *tiles);
mbc_status mbc_solver_get_factor_tiles(const mbc_solver *s, mbc_factor_tiles *tiles);
/* Autotuner: factor this solver `reps` times with each candidate tile shape
 * (class bounds first, then, for FP32 factors, the tensor-core threshold
 * tc_min_ns, then the panel rows of each class in turn, keeping the best so
 * far), time every factor with CUDA events on `stream`, and leave the
 * fastest shapes set on the solver.  best (optional) receives them and
 * ms_best (optional) the best factor time in ms.  The solver ends factored. */
mbc_status mbc_solver_tune_factor(mbc_solver *s, int32_t reps, mbc_factor_tiles *best,
                                  double *ms_best, mbc_stream stream);

/* Failure-path diagnostics: the number of polls after which a wait of the
 * tensor-core kernels (INT8 and 3xTF32 matvecs, tensor-core Gram) for a
 * partner role or a copy gives up (0: the default, 2^22).  On expiry the
 * kernel stops, waits with the default limit for its own copies and MMAs,
 * frees its tensor memory and returns; the call reports MBC_TIMEOUT and the
 * solver stays usable.  For tests: a small limit makes the waits expire. */
mbc_status mbc_solver_set_wait_limit(mbc_solver *s, uint32_t polls);

/* Number of supernodes of the last factor whose Theta_s was formed on the
 * tensor cores (mbc_factor_tiles.tc_min_ns). */
mbc_status mbc_solver_get_tensor_grams(const mbc_solver *s, int32_t *count);

/* Number of supernodes refactored in FP64 (FP32 solvers: cancelling or
 * non-positive pivots; FP64 solvers: the diagonal-shift retry). */
mbc_status mbc_solver_get_pivot_retries(const mbc_solver *s, int32_t *count);

typedef enum {
  MBC_MATVEC_AUTO = 0,   /* tensor cores for FP32 point-kernel matvecs with 8 <= R <= 256 */
  MBC_MATVEC_SIMT = 1,   /* CUDA-core kernels only */
  MBC_MATVEC_TENSOR = 2  /* tensor cores whenever R <= 256 (FP32 point kernel) */
} mbc_matvec_impl;

/* Choose the matvec implementation of an FP32 point-kernel solver (checks,
 * A/B timing).  Dense operators always use the CUDA-core kernels; FP64
 * matvecs follow mbc_solver_set_fp64_matvec. */
mbc_status mbc_solver_set_matvec(mbc_solver *s, int32_t impl);

typedef enum {
  MBC_FP64_MATVEC_SIMT = 0, /* FP64 CUDA-core kernels (the default) */
  MBC_FP64_MATVEC_INT8 = 1  /* FP64-accurate INT8 tensor-core matvec (exact digit slicing) */
} mbc_fp64_matvec;

/* Choose how the FP64 matvecs of a point-kernel solver run: the FP64 solve,
 * the FP64 residuals and polish of the mixed solve, and mbc_apply_K /
 * mbc_apply_KT of an FP64 solver.  The INT8 form stores G as five signed
 * 8-bit digit planes per direction, scaled by a power of two per row and
 * 2048-column chunk (2 x 5 x nf x n bytes of device memory), and forms the
 * products exactly in INT32 on the tensor cores.  An output is within
 * 2^-33 sum_chunks 2048 max|G| max|v| of the exact product (about 2e-10
 * relative on MFS operators).  The FP64 PCG then converges only on
 * residuals recomputed with the same operator.
 * Requested FP64 true residuals (true_residual option) always use the FP64
 * kernels.  The planes are built by mbc_solver_prepare or by the first call
 * that needs them; if the planes of every row do not fit, they are rebuilt
 * slab by slab for each matvec (MBC_NO_MEMORY if not even one slab fits).
 * After building, one column is checked against the FP64 kernels in both
 * directions (MBC_CUDA_ERROR if they differ by more than 1e-8 relative).
 * Dense operators: MBC_UNSUPPORTED. */
mbc_status mbc_solver_set_fp64_matvec(mbc_solver *s, int32_t impl);

/* Build the operator data the selected matvec implementations need (the INT8
 * digit planes) now, on `stream`, instead of inside the first solve. */
mbc_status mbc_solver_prepare(mbc_solver *s, mbc_stream stream);

typedef enum {
  MBC_SCHED_BATCHED = 0, /* all R columns advance together (per-column alpha, beta, stop) */
  MBC_SCHED_PER_RHS = 1, /* one cold-started PCG per column, in order (the reference's loop) */
  MBC_SCHED_BLOCK = 2    /* block PCG: all active columns share one Krylov space (FP64 recursions:
                            MBC_F64 solvers, or MBC_F32 with fp64_recursion; at most 512 columns);
                            every column still stops on its own residual */
} mbc_schedule;

typedef struct {
  int32_t max_iters;     /* per column (per refinement sweep in MBC_F32) */
  double tol;            /* stop when |r|^2 < tol^2 |b|^2, b = K^T f (kl_chol.cu:955) */
  int32_t schedule;      /* mbc_schedule */
  int32_t precondition;  /* 1 = KL preconditioner (the reference always passes true) */
  int32_t max_refine;    /* MBC_F32: max FP64 residual replacements (0 = plain FP32 PCG) */
  double inner_tol;      /* MBC_F32: replace once |r| fell by this factor since the last one */
  int32_t check_every;   /* iterations between convergence checks on the host */
  int32_t true_residual; /* 1 = report the FP64-recomputed |K^T(f-Kx)|/|K^T f| */
  int32_t profile;       /* 1 = time the matvec kernels with CUDA events on `stream` */
  int32_t graph;         /* 1 = replay blocks of check_every PCG iterations as a CUDA graph
                            (captured on the first full block; ignored with profile) */
  int32_t compact;       /* 1 = once at most half of the columns are still iterating (and at
                            least 8 have stopped), continue with those columns alone, so the
                            matvecs carry only them (FP64 and plain FP32 solves, and the
                            FP64 polish of MBC_F32 solves) */
  int32_t fp64_recursion; /* MBC_F32 solvers: run the whole PCG in FP64 (vectors, dot products,
                            scalars and the FP64 matvec chosen by mbc_solver_set_fp64_matvec),
                            keeping only the factor and its application in FP32; max_refine and
                            inner_tol are then unused.  Ignored by MBC_F64 solvers. */
} mbc_solve_options;

typedef struct {
  int32_t status_per_worst; /* worst per-column status */
  int32_t iters_max;        /* most iterations any column took */
  int64_t iters_total;      /* summed over columns */
  int32_t refinements;      /* outer sweeps done (MBC_F32) */
  int32_t n_converged;
  double relres_max;        /* recursive residual (or true one when requested) */
  double true_relres_max;   /* FP64 |K^T(f-Kx)|/|K^T f|, if requested, else -1 */
  double t_solve_ms;
  double t_matvec_ms;       /* profile: summed duration of the K and K^T kernels */
  int64_t n_matvec;         /* profile: K / K^T launches timed */
  int64_t kernel_launches;  /* kernels this call launched */
  int32_t n_polished;       /* MBC_F32: columns finished by FP64 PCG after the FP32
                               recursion stagnated or ran out of iterations */
  double t_matvec64_ms;     /* profile: the FP64 part of t_matvec_ms */
  int64_t n_matvec64;       /* profile: FP64 K / K^T launches timed */
  int64_t matvec64_columns; /* profile: columns summed over those launches (block PCG narrows) */
} mbc_solve_stats;

void mbc_solve_default_options(mbc_solve_options *opt);

/* Forward solve (kl_chol.cu:891-1088, per column of F):
 *   min |K x - f|  via  (K^T K) x = K^T f.
 * F: nf x R, X: n x R (ORIGINAL source order), element type f_dtype / x_dtype.
 * X0: NULL for a cold start (x0 = 0), else an n x R warm start (x_dtype).
 * iters_host: optional int32[R]. */
mbc_status mbc_solve(mbc_solver *s, int32_t R, const void *F, int32_t f_dtype, void *X,
                     int32_t x_dtype, const void *X0, const mbc_solve_options *opt,
                     mbc_solve_stats *stats_host, int32_t *iters_host, mbc_stream stream);

/* Adjoint solve (kl_chol.cu:1090-1264): (K^T K) x = b, B: n x R, ORIGINAL order. */
mbc_status mbc_solve_adjoint(mbc_solver *s, int32_t R, const void *B, int32_t b_dtype, void *X,
                             int32_t x_dtype, const mbc_solve_options *opt,
                             mbc_solve_stats *stats_host, int32_t *iters_host,
                             mbc_stream stream);

/* Operator applications in the ORIGINAL source order, for checks:
 * W (nf x R) = K V (n x R);  T (n x R) = K^T W.  dtype of V/W/T = precision. */
mbc_status mbc_apply_K(mbc_solver *s, int32_t R, const void *V, void *W, mbc_stream stream);
mbc_status mbc_apply_KT(mbc_solver *s, int32_t R, const void *W, void *T, mbc_stream stream);

/* Added-mass tensor and fluid forces of solved strengths: the consumer of the
 * solve in core/KTAB_Mfs_spclf1d.py:123-128 (phi = SL @ strengths,
 * Ks = Q @ phi * rho_fluid), with compute_single_layer and compute_quadrature
 * of utils/torch_utils.py:254-276, :336-347.  Point-kernel solvers only:
 *   phi(x_i, c) = sum_j X[j, c] / (4 pi |x_i - y_j|)               (FP64)
 *   Mf[6a + m, c] = -rho_fluid sum_{i in body a} w_i N_m(i) phi(x_i, c),
 *   N = (n, (x - centre_a) x n)   (the rigid-mode order of the right-hand sides).
 * The reference's SL is 1/|x - y| next to its solid-angle operator; with the
 * normal derivative of G = 1/(4 pi r) the same potential carries 1/(4 pi).
 * X: device n x R (x_dtype, ORIGINAL order); w: device nf float32 quadrature
 * weights; body_ptr: host int32[n_bodies + 1], rows of body a are
 * [body_ptr[a], body_ptr[a+1]); centers: host n_bodies x 3; Mf: host
 * (6 n_bodies) x R.  With accel (host double[R], R == 6 n_bodies) also
 * forces[6 n_bodies] = -Mf accel.  Synchronises the stream. */
mbc_status mbc_added_mass(mbc_solver *s, int32_t R, const void *X, int32_t x_dtype, const float *w,
                          int32_t n_bodies, const int32_t *body_ptr, const double *centers,
                          double rho_fluid, double *Mf, const double *accel, double *forces,
                          mbc_stream stream);

/* ------------------------------------------------------------------------ */
/* Warm-start network: a small MLP trained and evaluated on the GPU by this  */
/* library's own kernels.  No counterpart in the reference (its PCG always   */
/* starts from x0 = 0, kl_chol.cu:930-940): the network predicts a warm      */
/* start that the PCG then refines to the same FP64 true-residual criterion. */
/* Layers n_in -> hidden (tanh) x n_hidden_layers -> n_out (linear); BF16     */
/* weights in the products, FP32 accumulation, FP32 master weights + Adam.   */
/* Parameter vector layout: per layer W (row-major out x in), then b.        */
/* X, Y, T: device row-major batch x n_in / batch x n_out float32.          */
/* ------------------------------------------------------------------------ */
typedef struct mbc_mlp mbc_mlp;
mbc_status mbc_mlp_create(int32_t n_in, int32_t hidden, int32_t n_hidden_layers, int32_t n_out,
                          uint64_t seed, mbc_mlp **out);
mbc_status mbc_mlp_destroy(mbc_mlp *net);
mbc_status mbc_mlp_num_params(const mbc_mlp *net, int64_t *count);
mbc_status mbc_mlp_get_params(const mbc_mlp *net, float *params_host);
mbc_status mbc_mlp_set_params(mbc_mlp *net, const float *params_host);
mbc_status mbc_mlp_forward(mbc_mlp *net, int32_t batch, const float *X, float *Y, mbc_stream stream);
/* One step on the loss 0.5 mean((Y - T)^2): forward, backward and, for
 * lr > 0, an Adam update.  loss_host / grads_host (optional, host) receive
 * the batch loss and the gradient before the update. */
mbc_status mbc_mlp_train_step(mbc_mlp *net, int32_t batch, const float *X, const float *T, float lr,
                              double *loss_host, float *grads_host, mbc_stream stream);

/* Warm-start correction in the basis of the isolated-body solutions:
 *   X[j, 6b + m] += sum_k U[j, k] H[src_body[j]][b][k][m]
 * U: device n x 6 (each body's own rigid-mode solution on its sources),
 * H: device n_bodies x n_bodies x 6 x 6, X: device n x R float32 (ORIGINAL
 * order, R <= 6 n_bodies), src_body: device int32[n].  No counterpart in the
 * reference. */
mbc_status mbc_warm_correct(int32_t n, int32_t R, const int32_t *src_body, int32_t n_bodies,
                            const float *U, const float *H, float *X, mbc_stream stream);

/* Mesh collocation operator, assembled on the device: the collocation matrix
 * of a triangle-mesh scene, the solid angle of every face seen from every
 * source (utils/torch_utils.py:306-334, compute_solid_angle), and the
 * rigid-mode right-hand side FL @ IQ (core/KTAB_Mfs_spclf1d.py:101-111 with
 * utils/torch_utils.py:49-75), which the reference builds in torch each step:
 *   M[f, j] = 2 atan2(R1.(R2 x R3), l1 l2 l3 + (R1.R2) l3 + (R1.R3) l2 + (R2.R3) l1),
 *             Rk = V[F[f, k]] - S[j]          (n_faces x n_src, row stride ldm)
 *   rhs[f, 6b .. 6b+5] = (s, r x s) for face f of body b, zero elsewhere
 *             s = (v2 - v1) x (v3 - v1) / 2, r = face centre - body_pos[b]
 *             (n_faces x 6 n_bodies; rhs NULL to skip)
 * Computed in FP64 from float32 coordinates, stored as dtype (MBC_F32 for the
 * mfs_torch operator, or MBC_F64).  V: device n_vert x 3; F: device n_faces x 3
 * int32 vertex indices, counter-clockwise seen from outside; face_body: device
 * int32[n_faces]; body_pos: device n_bodies x 3; S: device n_src x 3.  A face
 * naming a vertex or body out of range gets NaN entries (nothing out of
 * bounds is read). */
mbc_status mbc_mesh_assemble(int32_t n_vert, const float *V, int32_t n_faces, const int32_t *F,
                             const int32_t *face_body, int32_t n_bodies, const float *body_pos,
                             int32_t n_src, const float *S, int32_t dtype, void *M, int64_t ldm,
                             void *rhs, mbc_stream stream);

/* Point-kernel matvec that allocates no device memory.  No counterpart in the
 * reference: it serves callers that cannot let a library call cudaMalloc or
 * cudaFree -- hosts that own the device through their own memory pool or a
 * fixed memory budget (a simulation loop, a framework's caching allocator),
 * where those calls can block on the whole device and fail late.
 *   transpose 0: out (nf x R) = coef K in (n x R),  K(i,j) = ((x_i - y_j) . nx_i) / |x_i - y_j|^3
 *   transpose 1: out (n x R)  = coef K^T in (nf x R)
 * x, nx: device nf x 3 float32; y: device n x 3 float32; in, out: device
 * row-major float32, ORIGINAL point order (no plan).  FP32 CUDA-core kernels.
 * Workspace: a 4 MiB static device array inside this library, held on every
 * GPU that loads it until exit; sizes with 2*ceil16(nf) + ceil16(n) > 262144
 * are refused with MBC_BAD_ARG.  The first call on a device looks the array's
 * address up (with that device current); make that first call before any
 * stream capture.  All calls share the array and each rewrites the parts it
 * reads, so calls whose kernels overlap on the GPU (different streams, or
 * several host threads) race: serialise them.  `in` and `out` must not
 * overlap (MBC_BAD_ARG).  A CUDA error already pending when the call starts is
 * returned as MBC_CUDA_ERROR and left pending.  The array's address is cached
 * per device: after cudaDeviceReset, do not call this again in the process. */
mbc_status mbc_point_apply_noalloc(int32_t transpose, int32_t nf, int32_t n, const float *x,
                                   const float *nx, const float *y, double coef, int32_t R,
                                   const float *in, float *out, mbc_stream stream);

/* ------------------------------------------------------------------------ */
/* mfs_torch operator bodies (the drop-in).                                   */
/* mbc_minvf_float replaces MinvF_float (mfs_torch/csrc/mfs_torch_ops.cu:21-197, */
/* registered as mfs_torch::MinvF_float_fastGrad, mfs_torch_ops.cpp:9);       */
/* mbc_vpl_fast_float replaces VpL_fast_float (mfs_torch_ops.cu:199-370,      */
/* mfs_torch_ops.cpp:8).  The context replaces the op's process-wide static  */
/* factor cache (mfs_torch_ops.cu:17-19): the adjoint reuses the factor of    */
/* the last forward on the same points and M, and refactors otherwise.        */
/*   M: device nf x n float32 row-major; F: device nf x R; pL: device n x R;  */
/*   Vs_host: host n x 3 float32; out: device n x R float32 (original order).  */
/* ------------------------------------------------------------------------ */
typedef struct mbc_context mbc_context;

mbc_status mbc_context_create(mbc_context **out);
mbc_status mbc_context_destroy(mbc_context *ctx);
/* Iterations / residual of the last call through this context. */
mbc_status mbc_context_last_stats(const mbc_context *ctx, mbc_solve_stats *stats_host);

mbc_status mbc_minvf_float(mbc_context *ctx, const float *M, int32_t nf, int32_t n,
                           const float *F, int32_t R, const float *Vs_host, double rho,
                           int64_t pcg_max_iter, double tol_r, int32_t timing_verbose,
                           int32_t solve_verbose, float *out, mbc_stream stream);

/* Gradients of MinvF_float_fastGrad (the reference's autograd,
 * core/mfs_torch_py/ops.py:42-58: grad_M = -M (W + W^T) + F LV, grad_F = M VpL,
 * W = A LV, LV = VpL^T) in low-rank form, without the N x N matrix W:
 *   G = M [A | VpL] (nf x 2R, into work), grad_F = M VpL,
 *   grad_M = (F - M A) VpL^T - (M VpL) A^T.
 * M: device nf x n float32 (row stride ldm); F: nf x R; A (the forward's
 * output) and VpL: n x R; work: device nf x 2R floats; grad_M (row stride ldg)
 * and grad_F may each be NULL to skip.  FP32 like the reference's products. */
mbc_status mbc_minvf_grad(int32_t nf, int32_t n, int32_t R, const float *M, int64_t ldm, const float *F,
                          const float *A, const float *VpL, float *work, float *grad_M, int64_t ldg,
                          float *grad_F, mbc_stream stream);

mbc_status mbc_vpl_fast_float(mbc_context *ctx, const float *M, int32_t nf, int32_t n,
                              const float *pL, int32_t R, const float *Vs_host, double rho,
                              int64_t pcg_max_iter, double tol_r, int32_t timing_verbose,
                              int32_t solve_verbose, float *out, mbc_stream stream);

#ifdef __cplusplus
}
#endif

#endif /* MBC_H */
