/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle of the vertex-patch Schwarz MG path.
 * Parity status: UNPINNED against the reference (no runnable reference, no
 * reference golden vectors); pinned against tests/golden/ fixtures computed
 * independently with numpy/scipy and against mathematical known answers.
 */
#ifndef TPS_ORACLE_H
#define TPS_ORACLE_H

#include <stddef.h>

#define ORC_MAXK 10
#define ORC_MAXN1 (2 * ORC_MAXK + 1)

#ifdef __cplusplus
extern "C" {
#endif

/* 1D finite-element data (oracle_fe.c) */
void orc_gauss(int nq, double *x, double *w);
void orc_gauss_lobatto(int k, double *x);
int orc_fe1d(int k, double *nodes, double *mass, double *lap, double *prol);
int orc_patch_matrices(int k, double *pmass, double *plap);
int orc_gen_eig(int m, const double *L, const double *M, double *V, double *lam);
int orc_patch_eigen(int k, double h, double *S, double *lam);

/* level operations, FP64 (_d) and FP32 (_f) (oracle_level.inc) */
#define ORC_LEVEL_DECL(SUF, REAL)                                                      \
  void orc_laplace_vmult##SUF(int dim, int k, int n, REAL *dst, const REAL *src,       \
                              const double *kappa);                                    \
  void orc_smoother_step##SUF(int dim, int k, int n, double omega, REAL *x,            \
                              const REAL *b, int zero_init, int reverse,               \
                              const double *kappa);                                    \
  void orc_prolongate_add##SUF(int dim, int k, int nc, REAL *fine, const REAL *coarse); \
  void orc_prolongate_add_nb##SUF(int dim, int k, int nc, REAL *fine, const REAL *coarse); \
  void orc_restrict_add##SUF(int dim, int k, int nc, REAL *coarse, const REAL *fine); \
  void orc_smoother_additive##SUF(int dim, int k, int n, double omega, REAL *x,        \
                                  const REAL *b, int zero_init);
ORC_LEVEL_DECL(_d, double)
ORC_LEVEL_DECL(_f, float)
#undef ORC_LEVEL_DECL

/* hierarchy + drivers (oracle_solve.c) */
typedef struct orc_hier orc_hier;
orc_hier *orc_hier_create(int dim, int k, int n_coarse, int n_levels, const double *kappa_fine);
void orc_hier_destroy(orc_hier *H);
long orc_hier_ndofs(const orc_hier *H, int level);
/* precision: 0 = FP64 V-cycle, 1 = FP32 V-cycle, 2 = FP64 V-cycle whose input
 * is rounded to FP32 precision first (the reference's "double" V-cycle). */
void orc_vcycle(orc_hier *H, int precision, int symmetric, double *dst, const double *src);
/* V-cycle smoothing on levels >= 1 by the additive step with damping omega
 * (on != 0) instead of the coloured multiplicative sweep (the coarse solve
 * is unchanged) */
void orc_hier_set_additive(orc_hier *H, int on, double omega);
void orc_vcycle_level(orc_hier *H, int precision, int symmetric, int level, double *dst,
                      const double *src);
void orc_fine_vmult(orc_hier *H, double *dst, const double *src);
/* flexible CG preconditioned by the V-cycle; returns iterations, fills history
 * with ||r_i||/||b|| (max_it+1 entries). */
int orc_solve_cg(orc_hier *H, int precision, int symmetric, const double *b, double *x,
                 double rel_tol, int max_it, double *history);
/* left-preconditioned GMRES with deal.II SolverGMRES semantics; returns the
 * iteration count, fills history with the preconditioned residual norms. */
int orc_solve_gmres(orc_hier *H, int precision, const double *b, double *x, double reduce,
                    double abs_tol, int max_it, int basis_size, double *history);
/* coarse direct solve of the hierarchy (interior DoFs, dense Cholesky) */
void orc_coarse_solve(orc_hier *H, double *dst, const double *src);
/* full multigrid pass (MultigridSolvers::solve): per-level right-hand sides,
 * optional per-level Dirichlet data (boundary entries used), finest solution */
void orc_fmg(orc_hier *H, int precision, int n_cycles, const double *const *rhs,
             const double *const *bnd, double *x);

#ifdef __cplusplus
}
#endif
#endif
