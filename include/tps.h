/*
 * tps.h -- C ABI of the B200-native vertex-patch Schwarz multigrid path
 * (continuous Q_k, uniform Cartesian meshes of the unit square/cube,
 * homogeneous Dirichlet boundary, lexicographic DoF numbering x fastest).
 *
 * Every entry point returns a tps_status; no C++ exception crosses the ABI.
 * Vectors are caller-owned DEVICE buffers of n_dofs(level) entries in the
 * lexicographic layout of the reference (include/utilities.cuh:44-100), the
 * element type given by `dtype`.  `stream` is a cudaStream_t (NULL = legacy
 * default stream).  A handle is not re-entrant: use one handle per host
 * thread / stream.
 */
#ifndef TPS_H
#define TPS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  TPS_OK = 0,
  TPS_ERR_INVALID = 1,      /* bad argument (null pointer, level, size, dtype) */
  TPS_ERR_CUDA = 2,         /* CUDA runtime/driver error */
  TPS_ERR_ALLOC = 3,        /* device or host allocation failed */
  TPS_ERR_NOT_CONVERGED = 4,/* solver hit max_iter before the tolerance */
  TPS_ERR_BREAKDOWN = 5,    /* Krylov breakdown (p^T A p <= 0, zero norm) */
  TPS_ERR_NONFINITE = 6,    /* NaN/Inf met in a residual or input */
  TPS_ERR_UNSUPPORTED = 7,  /* degree/dimension not compiled in */
  TPS_ERR_TIMEOUT = 8       /* a bounded device wait ran out (tps_device_status) */
} tps_status;

typedef enum {
  TPS_F64 = 0,
  TPS_F32 = 1,
  TPS_TF32 = 2, /* FP32 vectors; the 3D patch solves run on the tensor cores (TF32
                  operands, FP32 accumulation).  tps_smoother_step and
                  tps_time_smoother only. */
  TPS_TF32X3 = 3 /* as TPS_TF32 with every product formed from a three-term TF32
                    split (a_hi b_hi + a_hi b_lo + a_lo b_hi): about FP32 accuracy
                    per product, FP32 accumulation.  Degree 4 only. */
} tps_dtype;

typedef struct tps_handle tps_handle;

/* Problem description (replaces the reference's compile-time CT:: constants,
 * scripts/ct_parameter.py.in:109-124, and the DoFHandler/Triangulation set-up
 * of apps/poisson.cu:152-181). */
typedef struct {
  int dim;             /* 2 or 3 */
  int degree;          /* k, 1..7 */
  int n_coarse;        /* cells per direction of the coarsest level (>= 2) */
  int n_levels;        /* the finest level has n_coarse * 2^(n_levels-1) cells/direction */
  double relaxation;   /* smoother damping omega (reference default 1.0) */
  const double *kappa; /* HOST array of per-cell coefficients (> 0) on the finest
                          level (lexicographic cells) or NULL for kappa = 1 */
  int device;          /* CUDA device ordinal */
} tps_problem;

/* Lifecycle.  Replaces MultigridSolvers' constructor (include/solver.cuh:1545-1744):
 * builds every level's patch colouring, 1D matrices, FP64 eigendecompositions,
 * transfer data and the device work vectors. */
int tps_create(const tps_problem *problem, tps_handle **out);
int tps_destroy(tps_handle *h);
/* Message of the last failing call on `h` (or, when h is NULL, of the last
 * failing tps_create or tps_restrict_add_noalloc of this thread).  Valid until
 * the next call on the same handle/thread. */
const char *tps_last_error(const tps_handle *h);
/* Number of DoFs (boundary included) and cells per direction of `level`
 * (0 = coarsest, n_levels-1 = finest). */
int tps_level_info(const tps_handle *h, int level, int64_t *n_dofs, int *cells_per_dim);

/* LaplaceOperator::vmult (include/laplace_operator.cuh:86-101):
 * dst = A_level src on interior rows, dst = src on Dirichlet rows. */
int tps_laplace_vmult(tps_handle *h, int level, int dtype, void *dst, const void *src,
                      void *stream);

/* PatchSmoother::vmult / step (include/patch_smoother.cuh:155-292): one 2^d-coloured
 * multiplicative vertex-patch sweep x <- S(x, b); zero_init=1 is vmult (x := 0 first).
 * reverse=1 runs the colours in reverse order (symmetric post-smoothing). */
int tps_smoother_step(tps_handle *h, int level, int dtype, void *x, const void *b,
                      int zero_init, int reverse, void *stream);

/* The reference's other smoother variants (SmootherVariant GLOBAL, SEPERATE,
 * Exact; include/patch_base.cuh:28-90, dispatched in
 * PatchSmootherImpl::step_impl, include/patch_smoother.cuh:185-260), as
 * cross-checks of tps_smoother_step (TPS_SMOOTHER_FUSED).  Per colour the
 * residual r_I = (b - A x)_I is formed on the patch interiors -- per patch
 * from its box (SEPARATE, EXACT) or by the level operator (GLOBAL) -- into a
 * handle-owned vector, then x_I <- omega (x_I + A_II^{-1} r_I) per patch by
 * the fast diagonalisation (SEPARATE, GLOBAL) or by the dense inverse of the
 * assembled interior patch matrix (EXACT; computed in FP64 on the host at the
 * first EXACT call of a handle: (2k-1)^dim squared entries, 0.7 s on 8 host
 * threads for 3D Q7).  Same sweep as TPS_SMOOTHER_FUSED up to rounding.  dtype
 * TPS_F64 or TPS_F32; constant coefficient only (TPS_ERR_UNSUPPORTED with
 * kappa); lexicographic caller vectors. */
#define TPS_SMOOTHER_FUSED 0
#define TPS_SMOOTHER_SEPARATE 1
#define TPS_SMOOTHER_GLOBAL 2
#define TPS_SMOOTHER_EXACT 3
/* Additive vertex-patch Schwarz step (no reference counterpart: the reference
 * sweep is multiplicative; the benchmark's 2D configuration names the additive
 * form): x <- x + omega sum_p R_p^T A_p,II^{-1} R_p (b - A x), every patch's
 * residual from the same x, the handle's additive damping omega (see
 * tps_set_smoother_kind).  reverse is ignored; constant coefficient. */
#define TPS_SMOOTHER_ADDITIVE 4
int tps_smoother_step_variant(tps_handle *h, int level, int dtype, void *x, const void *b,
                              int zero_init, int reverse, int variant, void *stream);
/* Smoothing of the V-cycle's levels >= 1 (the coarse solve is unchanged):
 * TPS_SMOOTHER_FUSED (the default, the reference's coloured sweep) or
 * TPS_SMOOTHER_ADDITIVE with damping omega in [0, 2/2^dim) (the additive step
 * converges below 2/2^dim, since at most 2^dim patch colours overlap; 0
 * selects 1/2^dim).  Applies to later solves, V-cycles and FMG of this handle
 * and allocates the additive step's two scratch vectors. */
int tps_set_smoother_kind(tps_handle *h, int kind, double damping);

/* MGTransferCUDA::prolongate_and_add / restrict_and_add
 * (include/cuda_mg_transfer.template.cuh:575-671).  to_level / from_level is the
 * finer level (>= 1). */
int tps_prolongate_add(tps_handle *h, int to_level, int dtype, void *fine, const void *coarse,
                       void *stream);
int tps_restrict_add(tps_handle *h, int from_level, int dtype, void *coarse, const void *fine,
                     void *stream);

/* V-cycle precision. */
typedef enum {
  TPS_VCYCLE_F64 = 0,        /* FP64 V-cycle */
  TPS_VCYCLE_F32 = 1,        /* FP32 smoother/operator/transfer inside the V-cycle */
  TPS_VCYCLE_F64_ROUNDED = 2, /* FP64 V-cycle fed with FP32-rounded input: the
                                reference's "double" V-cycle (include/solver.cuh:64-78) */
  TPS_VCYCLE_TF32 = 3,        /* as TPS_VCYCLE_F32, with the 3D patch solves on the tensor
                                cores (TF32 operands, FP32 accumulation) on the levels
                                where that is faster: degrees 2..4, colours of at least
                                128 patches per multiprocessor; the other levels use the
                                FP32 smoother */
  TPS_VCYCLE_TF32X3 = 4       /* as TPS_VCYCLE_TF32 with the three-term TF32 split of
                                TPS_TF32X3 (FP32-accurate products) on the same levels,
                                degree 4 only; other degrees run TPS_VCYCLE_F32 */
} tps_vcycle_precision;

/* MultigridSolvers::vmult (include/solver.cuh:1915-1930): dst = V-cycle(src) on the
 * finest level, FP64 in and out. symmetric=1 post-smooths in reverse colour order. */
int tps_vcycle(tps_handle *h, int precision, int symmetric, double *dst, const double *src,
               void *stream);

typedef enum {
  TPS_DRIVER_CG = 0,    /* flexible CG, FP64 outer iteration (iterative refinement) */
  TPS_DRIVER_GMRES = 1  /* deal.II SolverGMRES semantics: left-preconditioned, basis 28,
                           convergence on the preconditioned residual (include/solver.cuh:1865-1910) */
} tps_driver;

typedef struct {
  int driver;          /* tps_driver */
  int precision;       /* tps_vcycle_precision */
  int symmetric;       /* reverse-order post-smoothing (CG default 1; GMRES parity 0) */
  int max_iter;        /* CG default 100; reference GMRES default 20 (MAX_STEPS_) */
  double rel_tol;      /* CG: ||b-Ax||/||b||; GMRES: reduction of the preconditioned residual */
  double abs_tol;      /* GMRES absolute tolerance (reference: 1e-16) */
  int use_graph;       /* capture one iteration as a CUDA graph (CG) */
} tps_solve_opts;

#define TPS_MAX_HISTORY 256
typedef struct {
  int iterations;
  int converged;
  double initial_residual;  /* ||r_0|| (CG: true residual; GMRES: preconditioned) */
  double final_residual;    /* relative to initial */
  double history[TPS_MAX_HISTORY]; /* relative residual per iteration, history[0] = 1 */
  double time_ms;           /* device time of the solve (CUDA events on the stream) */
} tps_report;

void tps_solve_opts_default(tps_solve_opts *opts);

/* Solve A x = b on the finest level.  b, x: DEVICE FP64 buffers (x holds the initial
 * guess on entry).  Replaces MultigridSolvers::solve_gmres and adds the MG-CG driver. */
int tps_solve(tps_handle *h, const tps_solve_opts *opts, const double *b, double *x,
              tps_report *report, void *stream);

/* MultigridSolvers::solve (include/solver.cuh:1784-1860): one full-multigrid
 * pass.  rhs[l] (level l = 0..n_levels-1, FP64 device vectors, lexicographic):
 * the right-hand side of every level, with the lifting of the Dirichlet data
 * already subtracted, as the reference assembles it on every level; bnd (may
 * be null): per level the Dirichlet values on the boundary DoFs (other entries
 * ignored).  Coarse solve plus one smoother step; then per level the coarse
 * solution with its Dirichlet data is prolongated without boundary
 * constraints (FP64), the fine boundary set to zero, the FP64 residual formed
 * and n_cycles V-cycles (precision: tps_vcycle_precision, reference colour
 * order) add the correction.  x (finest level) receives the solution with the
 * Dirichlet data on its boundary.  report (may be null): final_residual =
 * ||rhs - A x_0||/||rhs|| on the interior rows (x_0: x with zero boundary),
 * iterations = n_cycles, time_ms. */
int tps_fmg(tps_handle *h, int precision, int n_cycles, const double *const *rhs,
            const double *const *bnd, double *x, tps_report *report, void *stream);

/* Variable coefficient -div(kappa grad u) (no reference counterpart; the
 * reference's operator has kappa = 1).  A handle created with a kappa array can
 * change it: the finest-level values are replaced, the coarser levels take the
 * mean of their 2^d children; rebuild_coarse = 1 also refactors the dense
 * coarse solve (otherwise the V-cycle keeps its previous coarse operator, which
 * only affects the preconditioner).  Synchronises the device. */
int tps_set_kappa(tps_handle *h, const double *kappa_host, int rebuild_coarse);

/* dst = M src with the finest-level mass matrix (all rows), FP64, device
 * buffers.  Used for b = M f and the gradient dJ/df = M lambda. */
int tps_mass_vmult(tps_handle *h, double *dst, const double *src, void *stream);
/* Right-hand-side assembly on the device, the loop of
 * LaplaceOperator::compute_residual (include/laplace_operator.cuh:118-181, a
 * host loop over deal.II FEValues there) for a general f:
 * b_i = sum over the level's cells and their QGauss(k+1) points of
 * f(x_q) phi_i(x_q) JxW_q, Dirichlet rows zero.  f_quad (FP64 device array)
 * holds f at the Gauss points: cells lexicographic (x fastest), then the
 * (k+1)^dim points of the cell lexicographic (x fastest); the Gauss points of
 * [0,1] are those of orc_gauss/QGauss(k+1) mapped to the cell.  b: FP64,
 * lexicographic, n_dofs(level) entries.  Deterministic (cells added colour
 * by colour, no atomics). */
int tps_assemble_rhs(tps_handle *h, int level, const double *f_quad, double *b, void *stream);

/* Adjoint of the solve u = A(kappa)^{-1} M f for a loss J(u) (no reference
 * counterpart; the reference has no differentiable path): given the forward
 * solution u and g = dJ/du (FP64 device vectors, finest level,
 * lexicographic), solves A(kappa) lambda = g with the MG-preconditioned CG of
 * opts (driver TPS_DRIVER_CG; g's Dirichlet rows are taken as zero, so
 * lambda vanishes there) and returns
 *   dJdf[i]     = (M lambda)_i                      (all rows, as tps_mass_vmult)
 *   dJdkappa[c] = -lambda_c^T A_cell u_c per cell   (as -tps_cell_energy; may be
 *                 NULL, and needs a handle created with kappa)
 * report: the adjoint solve's.  Returns the adjoint solve's status (a gradient
 * of a solve that did not converge is returned with TPS_ERR_NOT_CONVERGED).
 * The handle keeps two more N-vectors between calls. */
int tps_adjoint(tps_handle *h, const tps_solve_opts *opts, const double *u, const double *g, double *dJdf,
                double *dJdkappa, tps_report *report, void *stream);

/* energy[c] = lambda_c^T A_cell u_c = int_c grad(lambda).grad(u) for every
 * finest-level cell c (lexicographic cells), FP64: dJ/dkappa_c = -energy[c]
 * for J(u(kappa)) with adjoint state lambda. */
int tps_cell_energy(tps_handle *h, const double *u, const double *lam, double *energy,
                    void *stream);

/* Measurement hook: runs `sweeps` coloured sweeps of the level's smoother on
 * the V-cycle's own work vectors (the padded, TMA-staged path that the V-cycle
 * uses) on `stream` and returns the mean device time of one sweep (CUDA events
 * on that stream).  Used by the benchmark to time the dominant kernel. */
int tps_time_smoother(tps_handle *h, int level, int dtype, int sweeps, double *ms_per_sweep,
                      void *stream);

/* Same solve with HOST buffers; the host<->device copies are part of the call.
 * The handle keeps two device staging vectors (16 N bytes) between calls. */
int tps_solve_host(tps_handle *h, const tps_solve_opts *opts, const double *b_host,
                   double *x_host, tps_report *report);
/* The same with a separate initial guess: x0_host (N entries, may equal
 * x_host) is copied in, or, when NULL, the solve starts from x = 0 on the
 * device without a host-to-device copy of the guess; the solution is written
 * to x_host.  tps_solve_host(h, o, b, x, r) is this call with x0_host = x. */
int tps_solve_host_guess(tps_handle *h, const tps_solve_opts *opts, const double *b_host,
                         const double *x0_host, double *x_host, tps_report *report);
/* n solves of the same system with HOST right-hand sides b_host[i] and
 * solutions x_host[i] (N entries each, every solve from x = 0), one after the
 * other, with the copies overlapped with the solves: b[i+1] is copied in and
 * x[i-1] out while solve i runs, on a second stream.  Overlap needs pinned
 * host buffers (cudaHostAlloc / cudaHostRegister); pageable ones give the same
 * results without it.  reports[i] per solve; x_host[i] is written when solve i
 * returns TPS_OK or TPS_ERR_NOT_CONVERGED.  The return value is TPS_OK when
 * every solve converged, else the first failure (a non-convergence only when
 * nothing worse happened).  The handle keeps 5 more device vectors (40 N bytes)
 * between calls.  No counterpart in the reference (a host loop over
 * tps_solve_host_guess, without the overlap). */
int tps_solve_host_many(tps_handle *h, const tps_solve_opts *opts, int n, const double *const *b_host,
                        double *const *x_host, tps_report *reports);

/* Autotuner of the 3D level kernels (the reference's
 * AdditionalData::patch_per_block, include/patch_smoother.cuh:101-118, fixed
 * there, chosen here by timing): on every level of the dtype's V-cycle it times
 * each compiled smoother variant (patches per CTA batch, one warp per patch,
 * two patches per warp) and each tile depth of the operator (1, 2, 4, 8 or
 * 16 cell layers per CTA of the z-marching kernel), and keeps the fastest of each
 * for later sweeps, operator applications and V-cycles of this handle.
 * ppb_per_level (n_levels entries, may be null) receives the chosen smoother
 * values (0 in 2D, -1 for one warp per patch, -2 for two patches per warp).
 * Batched solves tune their systems automatically. */
int tps_autotune(tps_handle *h, int dtype, int *ppb_per_level);
/* The operator tile depth a level of the dtype's V-cycle uses: the cell layers
 * per CTA that tps_autotune chose, or 0 for the library's rule (16 layers, fewer
 * where a level would have fewer than 148 CTAs). */
int tps_get_operator_layers(tps_handle *h, int dtype, int level, int *layers);
/* Set the operator tile depth of a level explicitly (1, 2, 4, 8 or 16 cell
 * layers per CTA; 0 restores the library's rule).  The mat-vec is bit-identical for
 * every depth; the fused p.q of the outer CG is summed per CTA, so a solve's
 * rounding follows the depth of the finest level. */
int tps_set_operator_layers(tps_handle *h, int dtype, int level, int layers);
/* The compiled variants of the 3D smoother, TPS_SMOOTHER_VARIANTS entries:
 * patches per CTA batch 0 default, 1 half, 2 quarter, 3 one warp per patch
 * (reported as -1 where it is compiled) and 4 two patches per warp in packed
 * FP32 arithmetic (FP32 only, degrees 2..5; reported as -2 where it is
 * compiled); a variant that is not compiled reports variant 0's value, and
 * 2D reports 0.  tps_set_smoother_variant makes the explicit choice of one
 * for a level (what tps_autotune sets).  All variants give bit-identical
 * sweeps. */
#define TPS_SMOOTHER_VARIANTS 5
int tps_smoother_variants(tps_handle *h, int dtype, int *ppb);
int tps_set_smoother_variant(tps_handle *h, int dtype, int level, int variant);
/* The variant a level's sweeps use now: the one set or autotuned, else the
 * library default, the fastest measured per level size.
 * FP32:
 *   - two patches per warp where a colour holds at least 4096 patches
 *     (degrees 2..4), and at degree 4 from 512 patches;
 *   - one warp per patch at degree 2 from 512 patches;
 *   - otherwise the default CTA batch on large levels and half batches on
 *     smaller ones.
 * FP64:
 *   - one warp per patch at degree 4, and at degree 3 where a colour holds
 *     at least 4096 patches;
 *   - otherwise quarter CTA batches at degrees 2 and 3, and the default batch
 *     at other degrees. */
int tps_get_smoother_variant(tps_handle *h, int dtype, int level, int *variant);

/* ---- batched solves (no reference counterpart) ----------------------------
 * A batch owns n independent systems (1 <= n <= 256): right-hand sides of one
 * mesh and/or meshes of different sizes; system i is built from problems[i]
 * with its own hierarchy and work vectors.  tps_batch_solve runs the MG-CG of
 * every system as ONE CUDA graph launch: the initial residuals on parallel
 * branches, then a device-side while loop (a conditional graph node) whose body
 * runs one CG iteration of every system that is still iterating (one
 * conditional node per system, parallel branches) followed by a check kernel;
 * the host waits once, when every system has converged or reached max_iter.
 * The instantiated graph is reused while opts, stream and the vector pointers
 * stay the same. */
typedef struct tps_batch tps_batch;
int tps_batch_create(const tps_problem *problems, int n_systems, tps_batch **out);
int tps_batch_destroy(tps_batch *b);
const char *tps_batch_last_error(const tps_batch *b);
/* the handle of system i (owned by the batch): level operations, tps_level_info */
int tps_batch_system(tps_batch *b, int i, tps_handle **h);
/* rhs[i], x[i]: DEVICE FP64 vectors of system i (x[i] holds the initial guess);
 * reports[i] per system (time_ms: the whole batch).  Driver must be TPS_DRIVER_CG;
 * use_graph is implied.  Returns TPS_OK when every system converged. */
int tps_batch_solve(tps_batch *b, const tps_solve_opts *opts, const double *const *rhs,
                    double *const *x, tps_report *reports, void *stream);

/* coarse += R fine, like tps_restrict_add, without a handle and without any
 * device allocation, for callers that must not allocate device memory (their
 * framework owns it all, e.g. a caching allocator or a pre-reserved arena).
 * No counterpart in the reference.  The 3D intermediate lives in a fixed
 * 16 MiB array inside the library (held on every GPU that loads it until the
 * process exits); 8 * (2n_c k+1) * (n_c k+1)^2 bytes (FP64; half for FP32)
 * must fit, larger sizes return TPS_ERR_INVALID.  n_coarse_cells: cells per
 * direction of the coarse level; vectors lexicographic.  The first call on a
 * device (and the first one after the device's context was reset, e.g. by
 * cudaDeviceReset) uploads the 1D tables to constant memory: make it before
 * any stream capture.  Every call looks the array's address up in the current
 * context.  Calls share the array: calls that overlap on the GPU race. */
int tps_restrict_add_noalloc(int dim, int degree, int n_coarse_cells, int dtype, void *coarse,
                             const void *fine, void *stream);

/* Failure detection (no counterpart in the reference).  Every device wait of
 * the library is bounded: the 3D smoothers wait for their TMA stages for at
 * most ~2^31 SM cycles, then record the timeout in a flag of the handle and
 * return instead of spinning.  tps_solve, tps_solve_host(_guess), tps_fmg,
 * tps_time_smoother and tps_batch_solve read the flag once their stream's work
 * is done, clear it and return TPS_ERR_TIMEOUT when it was set (the results of
 * the call are then invalid).  The asynchronous level calls leave it set:
 * tps_device_status synchronizes the device, reads and clears it and returns
 * TPS_ERR_TIMEOUT or TPS_OK. */
int tps_device_status(tps_handle *h);
/* Runs the error path of a bounded wait without any fault: one CTA waits, with
 * the smoothers' wait loop, on an mbarrier that nothing arrives on, gives up
 * after `cycles` SM cycles (1 .. 2^31) and records the timeout in the handle's
 * flag like a smoother launch would.  Asynchronous on `stream`. */
int tps_selftest_wait_timeout(tps_handle *h, long long cycles, void *stream);
/* Host self-check of the 2^dim colouring (no device work): on a level of
 * n_cells per direction, every interior vertex is the centre of exactly one
 * patch, the interiors of one colour's patches are disjoint, and no patch's
 * box ring (read while the colour runs) meets another patch's interior
 * (written) -- the race freedom of the in-place colour sweep, which the
 * reference asserts only for the colour sizes in debug builds
 * (include/patch_base.template.cuh:1279-1284).  TPS_OK, or TPS_ERR_INVALID
 * with the first violation in tps_last_error(NULL). */
int tps_check_colouring(int dim, int degree, int n_cells);
/* Testing hook: the n-th device allocation of the library from now (n >= 1,
 * counted over all handles and batches of the process) fails as cudaMalloc does
 * on a full device, so the calls report TPS_ERR_ALLOC; n = 0 disarms it. */
void tps_inject_alloc_failure(int n);

#ifdef __cplusplus
}
#endif
#endif
