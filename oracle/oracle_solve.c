/*
 * TEST INFRASTRUCTURE ONLY -- MG hierarchy, V-cycle and Krylov drivers of the
 * CPU oracle.  Parity status: UNPINNED (see oracle.h).
 *
 *  - V-cycle: MultigridSolvers::v_cycle (include/solver.cuh:1952-2001):
 *    pre-smooth with zero initial guess (smoother vmult), t = d - A su,
 *    restrict, recurse, prolongate-and-add, post-smooth (step).  The coarsest
 *    level of a 2-cell mesh is the single-patch smoother (exact local solve,
 *    include/solver.cuh:80-102 and :1958-1965); other coarse meshes use a dense
 *    FP64 Cholesky solve (no reference counterpart).
 *  - The V-cycle entry converts FP64 -> V-cycle precision as
 *    copy_vector<true> does (include/solver.cuh:64-78, :1915-1930); precision
 *    mode 2 reproduces the reference's rounding of the "double" V-cycle input
 *    through __double2float_rn.
 *  - GMRES: deal.II SolverGMRES defaults as used by solve_gmres
 *    (include/solver.cuh:1865-1910): left preconditioning, Arnoldi basis of
 *    max_n_tmp_vectors-2 = 28 vectors, modified Gram-Schmidt, Givens
 *    rotations, convergence on the preconditioned residual estimate with
 *    ReductionControl(max_steps, abs_tol, reduce).
 *  - CG: flexible (Polak-Ribiere) CG on the true FP64 residual; no reference
 *    counterpart (the reference's driver is GMRES).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

struct orc_hier {
  int dim, k, n_coarse, n_levels;
  int *n;           /* cells per direction per level */
  long *N;          /* DoFs per level */
  double **kappa;   /* per level, NULL if constant coefficient */
  double *d64[3];   /* scratch per level group: allocated per level below */
  double **dd, **sud, **td;  /* FP64 V-cycle vectors */
  float **df, **suf, **tf;   /* FP32 V-cycle vectors */
  int additive;       /* additive smoothing on levels >= 1 */
  double add_omega;
  /* dense coarse factor */
  int use_dense_coarse;
  long n_int_coarse;
  long *coarse_int_idx;
  double *coarse_L;
};

static long ipow_l(long b, int e)
{
  long r = 1;
  while (e-- > 0) r *= b;
  return r;
}

static int is_boundary(int dim, int N1, long i)
{
  int x = (int)(i % N1), y = (int)((i / N1) % N1), z = dim == 3 ? (int)(i / ((long)N1 * N1)) : 0;
  return x == 0 || x == N1 - 1 || y == 0 || y == N1 - 1 || (dim == 3 && (z == 0 || z == N1 - 1));
}

void orc_hier_set_additive(orc_hier *H, int on, double omega)
{
  H->additive = on;
  H->add_omega = omega;
}

orc_hier *orc_hier_create(int dim, int k, int n_coarse, int n_levels, const double *kappa_fine)
{
  if ((dim != 2 && dim != 3) || k < 1 || k > ORC_MAXK || n_coarse < 2 || n_levels < 1) return NULL;
  orc_hier *H = (orc_hier *)calloc(1, sizeof(orc_hier));
  H->dim = dim;
  H->k = k;
  H->n_coarse = n_coarse;
  H->n_levels = n_levels;
  H->n = (int *)calloc(n_levels, sizeof(int));
  H->N = (long *)calloc(n_levels, sizeof(long));
  H->kappa = (double **)calloc(n_levels, sizeof(double *));
  H->dd = (double **)calloc(n_levels, sizeof(double *));
  H->sud = (double **)calloc(n_levels, sizeof(double *));
  H->td = (double **)calloc(n_levels, sizeof(double *));
  H->df = (float **)calloc(n_levels, sizeof(float *));
  H->suf = (float **)calloc(n_levels, sizeof(float *));
  H->tf = (float **)calloc(n_levels, sizeof(float *));
  for (int l = 0; l < n_levels; ++l) {
    H->n[l] = n_coarse << l;
    H->N[l] = ipow_l((long)H->n[l] * k + 1, dim);
    H->dd[l] = (double *)calloc(H->N[l], sizeof(double));
    H->sud[l] = (double *)calloc(H->N[l], sizeof(double));
    H->td[l] = (double *)calloc(H->N[l], sizeof(double));
    H->df[l] = (float *)calloc(H->N[l], sizeof(float));
    H->suf[l] = (float *)calloc(H->N[l], sizeof(float));
    H->tf[l] = (float *)calloc(H->N[l], sizeof(float));
  }
  if (kappa_fine) {
    /* coarse-level coefficients: mean of the 2^dim children */
    int L = n_levels - 1;
    long nc = ipow_l(H->n[L], dim);
    H->kappa[L] = (double *)malloc(sizeof(double) * nc);
    memcpy(H->kappa[L], kappa_fine, sizeof(double) * nc);
    for (int l = L - 1; l >= 0; --l) {
      int n = H->n[l], nf = H->n[l + 1];
      long ncl = ipow_l(n, dim);
      H->kappa[l] = (double *)calloc(ncl, sizeof(double));
      for (long c = 0; c < ncl; ++c) {
        int cx = (int)(c % n), cy = (int)((c / n) % n), cz = dim == 3 ? (int)(c / ((long)n * n)) : 0;
        double s = 0;
        for (int q = 0; q < (1 << dim); ++q) {
          int fx = 2 * cx + (q & 1), fy = 2 * cy + ((q >> 1) & 1), fz = 2 * cz + ((q >> 2) & 1);
          long fi = fx + (long)fy * nf + (dim == 3 ? (long)fz * nf * nf : 0);
          s += H->kappa[l + 1][fi];
        }
        H->kappa[l][c] = s / (1 << dim);
      }
    }
  }
  H->use_dense_coarse = (n_coarse != 2) || (kappa_fine != NULL);
  if (H->use_dense_coarse) {
    const int N1 = n_coarse * k + 1;
    const long Nc = H->N[0];
    long ni = 0;
    H->coarse_int_idx = (long *)malloc(sizeof(long) * Nc);
    for (long i = 0; i < Nc; ++i)
      if (!is_boundary(dim, N1, i)) H->coarse_int_idx[ni++] = i;
    H->n_int_coarse = ni;
    double *A = (double *)calloc((size_t)ni * ni, sizeof(double));
    double *e = (double *)calloc(Nc, sizeof(double));
    double *y = (double *)calloc(Nc, sizeof(double));
    for (long j = 0; j < ni; ++j) {
      e[H->coarse_int_idx[j]] = 1.0;
      orc_laplace_vmult_d(dim, k, n_coarse, y, e, H->kappa[0]);
      for (long i = 0; i < ni; ++i) A[i * ni + j] = y[H->coarse_int_idx[i]];
      e[H->coarse_int_idx[j]] = 0.0;
    }
    /* Cholesky, lower triangle */
    for (long j = 0; j < ni; ++j) {
      double s = A[j * ni + j];
      for (long p = 0; p < j; ++p) s -= A[j * ni + p] * A[j * ni + p];
      A[j * ni + j] = sqrt(s);
      for (long i = j + 1; i < ni; ++i) {
        double t = A[i * ni + j];
        for (long p = 0; p < j; ++p) t -= A[i * ni + p] * A[j * ni + p];
        A[i * ni + j] = t / A[j * ni + j];
      }
    }
    H->coarse_L = A;
    free(e);
    free(y);
  }
  return H;
}

void orc_hier_destroy(orc_hier *H)
{
  if (!H) return;
  for (int l = 0; l < H->n_levels; ++l) {
    free(H->kappa[l]);
    free(H->dd[l]);
    free(H->sud[l]);
    free(H->td[l]);
    free(H->df[l]);
    free(H->suf[l]);
    free(H->tf[l]);
  }
  free(H->kappa);
  free(H->dd);
  free(H->sud);
  free(H->td);
  free(H->df);
  free(H->suf);
  free(H->tf);
  free(H->n);
  free(H->N);
  free(H->coarse_int_idx);
  free(H->coarse_L);
  free(H);
}

long orc_hier_ndofs(const orc_hier *H, int level) { return H->N[level]; }

void orc_coarse_solve(orc_hier *H, double *dst, const double *src)
{
  const long ni = H->n_int_coarse, Nc = H->N[0];
  const double *A = H->coarse_L;
  double *y = (double *)malloc(sizeof(double) * ni);
  for (long i = 0; i < ni; ++i) {
    double t = src[H->coarse_int_idx[i]];
    for (long p = 0; p < i; ++p) t -= A[i * ni + p] * y[p];
    y[i] = t / A[i * ni + i];
  }
  for (long i = ni - 1; i >= 0; --i) {
    double t = y[i];
    for (long p = i + 1; p < ni; ++p) t -= A[p * ni + i] * y[p];
    y[i] = t / A[i * ni + i];
  }
  memset(dst, 0, sizeof(double) * Nc);
  for (long i = 0; i < ni; ++i) dst[H->coarse_int_idx[i]] = y[i];
  free(y);
}

#define DEFINE_VCYCLE(SUF, REAL, D, SU, T)                                                \
  static void vcycle_rec##SUF(orc_hier *H, int symmetric, int l, int zero_init)          \
  {                                                                                       \
    const int dim = H->dim, k = H->k;                                                     \
    if (l == 0) {                                                                         \
      if (!H->use_dense_coarse) {                                                         \
        orc_smoother_step##SUF(dim, k, H->n[0], 1.0, H->SU[0], H->D[0], 1, 0, H->kappa[0]); \
      } else {                                                                            \
        long N0 = H->N[0];                                                                \
        double *s = (double *)calloc((size_t)(N0 > 0 ? N0 : 1), sizeof(double));          \
        double *o = (double *)malloc(sizeof(double) * (size_t)(N0 > 0 ? N0 : 1));         \
        for (long i = 0; i < N0; ++i) s[i] = H->D[0][i];                                  \
        orc_coarse_solve(H, o, s);                                                        \
        for (long i = 0; i < N0; ++i) H->SU[0][i] = (REAL)o[i];                           \
        free(s);                                                                          \
        free(o);                                                                          \
      }                                                                                   \
      return;                                                                             \
    }                                                                                     \
    const int n = H->n[l];                                                                \
    const long N = H->N[l];                                                               \
    if (H->additive)                                                                      \
      orc_smoother_additive##SUF(dim, k, n, H->add_omega, H->SU[l], H->D[l], zero_init);  \
    else                                                                                  \
      orc_smoother_step##SUF(dim, k, n, 1.0, H->SU[l], H->D[l], zero_init, 0, H->kappa[l]); \
    orc_laplace_vmult##SUF(dim, k, n, H->T[l], H->SU[l], H->kappa[l]);                    \
    for (long i = 0; i < N; ++i) H->T[l][i] = H->D[l][i] - H->T[l][i];                    \
    memset(H->D[l - 1], 0, sizeof(REAL) * H->N[l - 1]);                                   \
    orc_restrict_add##SUF(dim, k, H->n[l - 1], H->D[l - 1], H->T[l]);                     \
    vcycle_rec##SUF(H, symmetric, l - 1, 1);                                              \
    orc_prolongate_add##SUF(dim, k, H->n[l - 1], H->SU[l], H->SU[l - 1]);                 \
    if (H->additive)                                                                      \
      orc_smoother_additive##SUF(dim, k, n, H->add_omega, H->SU[l], H->D[l], 0);          \
    else                                                                                  \
      orc_smoother_step##SUF(dim, k, n, 1.0, H->SU[l], H->D[l], 0, symmetric, H->kappa[l]); \
  }

DEFINE_VCYCLE(_d, double, dd, sud, td)
DEFINE_VCYCLE(_f, float, df, suf, tf)

void orc_vcycle_level(orc_hier *H, int precision, int symmetric, int level, double *dst,
                      const double *src)
{
  const long N = H->N[level];
  if (precision == 1) {
    for (long i = 0; i < N; ++i) H->df[level][i] = (float)src[i];
    vcycle_rec_f(H, symmetric, level, 1);
    for (long i = 0; i < N; ++i) dst[i] = (double)H->suf[level][i];
  } else {
    for (long i = 0; i < N; ++i)
      H->dd[level][i] = precision == 2 ? (double)(float)src[i] : src[i];
    vcycle_rec_d(H, symmetric, level, 1);
    memcpy(dst, H->sud[level], sizeof(double) * N);
  }
}

void orc_vcycle(orc_hier *H, int precision, int symmetric, double *dst, const double *src)
{
  orc_vcycle_level(H, precision, symmetric, H->n_levels - 1, dst, src);
}

/* MultigridSolvers::solve (include/solver.cuh:1784-1860): coarse solve plus
 * one smoother step, then per finer level: Dirichlet data on the coarse
 * solution, prolongation without boundary constraints (FP64), fine boundary
 * set to zero, FP64 residual, n_cycles V-cycles in the V-cycle precision
 * (v_cycle(level, n_cycles): the first pre-smoothing starts from zero, later
 * ones continue), correction added.  The solution is kept with zero boundary
 * entries (the Dirichlet data enter through the lifting in rhs) and the data
 * are written into the boundary of x at the end (get_solution, :1776-1781). */
void orc_fmg(orc_hier *H, int precision, int n_cycles, const double *const *rhs,
             const double *const *bnd, double *x)
{
  const int L = H->n_levels - 1, dim = H->dim, k = H->k;
  double **sol = (double **)calloc(L + 1, sizeof(double *));
  for (int l = 0; l < L; ++l) sol[l] = (double *)calloc(H->N[l], sizeof(double));
  sol[L] = x;
  double *res = (double *)malloc(sizeof(double) * H->N[L]);
  /* coarse level: coarse solve, then one more smoother step */
  {
    const long N0 = H->N[0];
    if (precision == 1) {
      for (long i = 0; i < N0; ++i) H->df[0][i] = (float)rhs[0][i];
      vcycle_rec_f(H, 0, 0, 1);
      orc_smoother_step_f(dim, k, H->n[0], 1.0, H->suf[0], H->df[0], 0, 0, H->kappa[0]);
      for (long i = 0; i < N0; ++i) sol[0][i] = (double)H->suf[0][i];
    } else {
      for (long i = 0; i < N0; ++i) H->dd[0][i] = rhs[0][i];
      vcycle_rec_d(H, 0, 0, 1);
      orc_smoother_step_d(dim, k, H->n[0], 1.0, H->sud[0], H->dd[0], 0, 0, H->kappa[0]);
      memcpy(sol[0], H->sud[0], sizeof(double) * N0);
    }
  }
  for (int l = 1; l <= L; ++l) {
    const long Nc = H->N[l - 1], N = H->N[l];
    const int N1c = H->n[l - 1] * k + 1, N1 = H->n[l] * k + 1;
    if (bnd && bnd[l - 1])
      for (long i = 0; i < Nc; ++i)
        if (is_boundary(dim, N1c, i)) sol[l - 1][i] = bnd[l - 1][i];
    memset(sol[l], 0, sizeof(double) * N);
    orc_prolongate_add_nb_d(dim, k, H->n[l - 1], sol[l], sol[l - 1]);
    if (bnd && bnd[l - 1])
      for (long i = 0; i < Nc; ++i)
        if (is_boundary(dim, N1c, i)) sol[l - 1][i] = 0.0;
    orc_laplace_vmult_d(dim, k, H->n[l], res, sol[l], H->kappa[l]);
    for (long i = 0; i < N; ++i) res[i] = is_boundary(dim, N1, i) ? 0.0 : rhs[l][i] - res[i];
    for (int c = 0; c < n_cycles; ++c) {
      if (precision == 1) {
        for (long i = 0; i < N; ++i) H->df[l][i] = (float)res[i];
        vcycle_rec_f(H, 0, l, c == 0);
      } else {
        for (long i = 0; i < N; ++i) H->dd[l][i] = res[i];
        vcycle_rec_d(H, 0, l, c == 0);
      }
    }
    if (precision == 1)
      for (long i = 0; i < N; ++i) sol[l][i] += (double)H->suf[l][i];
    else
      for (long i = 0; i < N; ++i) sol[l][i] += H->sud[l][i];
  }
  if (bnd && bnd[L])
    for (long i = 0; i < H->N[L]; ++i)
      if (is_boundary(dim, H->n[L] * k + 1, i)) x[i] = bnd[L][i];
  for (int l = 0; l < L; ++l) free(sol[l]);
  free(sol);
  free(res);
}

void orc_fine_vmult(orc_hier *H, double *dst, const double *src)
{
  int L = H->n_levels - 1;
  orc_laplace_vmult_d(H->dim, H->k, H->n[L], dst, src, H->kappa[L]);
}

static double dot(long n, const double *a, const double *b)
{
  double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (long i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

int orc_solve_cg(orc_hier *H, int precision, int symmetric, const double *b, double *x,
                 double rel_tol, int max_it, double *history)
{
  const long N = H->N[H->n_levels - 1];
  double *r = (double *)malloc(sizeof(double) * N), *z = (double *)malloc(sizeof(double) * N);
  double *p = (double *)malloc(sizeof(double) * N), *q = (double *)malloc(sizeof(double) * N);
  orc_fine_vmult(H, q, x);
  for (long i = 0; i < N; ++i) r[i] = b[i] - q[i];
  const double bnorm = sqrt(dot(N, b, b));
  double res = sqrt(dot(N, r, r)) / (bnorm > 0 ? bnorm : 1.0);
  if (history) history[0] = res;
  int it = 0;
  if (res > rel_tol) {
    orc_vcycle(H, precision, symmetric, z, r);
    memcpy(p, z, sizeof(double) * N);
    double rz = dot(N, r, z);
    for (it = 1; it <= max_it; ++it) {
      orc_fine_vmult(H, q, p);
      double alpha = rz / dot(N, p, q);
      for (long i = 0; i < N; ++i) {
        x[i] += alpha * p[i];
        r[i] -= alpha * q[i];
      }
      res = sqrt(dot(N, r, r)) / (bnorm > 0 ? bnorm : 1.0);
      if (history) history[it] = res;
      if (res <= rel_tol) break;
      orc_vcycle(H, precision, symmetric, z, r);
      /* flexible beta: z_new . (r_new - r_old) / rz, with r_new - r_old = -alpha q */
      double beta = -alpha * dot(N, z, q) / rz;
      rz = dot(N, r, z);
      for (long i = 0; i < N; ++i) p[i] = z[i] + beta * p[i];
    }
    if (it > max_it) it = max_it;
  }
  free(r);
  free(z);
  free(p);
  free(q);
  return it;
}

int orc_solve_gmres(orc_hier *H, int precision, const double *b, double *x, double reduce,
                    double abs_tol, int max_it, int basis_size, double *history)
{
  const long N = H->N[H->n_levels - 1];
  const int m = basis_size;
  double **V = (double **)malloc(sizeof(double *) * (m + 1));
  for (int i = 0; i <= m; ++i) V[i] = (double *)malloc(sizeof(double) * N);
  double *p = (double *)malloc(sizeof(double) * N);
  double *Hm = (double *)calloc((size_t)(m + 1) * m, sizeof(double));
  double *h = (double *)calloc(m + 1, sizeof(double));
  double *gam = (double *)calloc(m + 1, sizeof(double));
  double *ci = (double *)calloc(m + 1, sizeof(double));
  double *si = (double *)calloc(m + 1, sizeof(double));
  int acc = 0, state = 0; /* 0 iterate, 1 success, 2 failure */
  double tol = abs_tol;
  do {
    orc_fine_vmult(H, p, x);
    for (long i = 0; i < N; ++i) p[i] = b[i] - p[i];
    orc_vcycle(H, precision, 0, V[0], p);
    double rho = sqrt(dot(N, V[0], V[0]));
    /* ReductionControl::check at step acc */
    if (acc == 0) tol = fmax(abs_tol, reduce * rho);
    if (history) history[acc] = rho;
    if (rho <= tol) { state = 1; break; }
    if (acc >= max_it) { state = 2; break; }
    gam[0] = rho;
    for (long i = 0; i < N; ++i) V[0][i] /= rho;
    int dimk = 0;
    for (int inner = 0; inner < m && state == 0; ++inner) {
      ++acc;
      orc_fine_vmult(H, p, V[inner]);
      orc_vcycle(H, precision, 0, V[inner + 1], p);
      dimk = inner + 1;
      /* modified Gram-Schmidt */
      for (int i = 0; i < dimk; ++i) {
        h[i] = dot(N, V[inner + 1], V[i]);
        for (long j = 0; j < N; ++j) V[inner + 1][j] -= h[i] * V[i][j];
      }
      double s = sqrt(dot(N, V[inner + 1], V[inner + 1]));
      h[inner + 1] = s;
      if (s != 0)
        for (long j = 0; j < N; ++j) V[inner + 1][j] /= s;
      /* Givens rotations */
      for (int i = 0; i < inner; ++i) {
        double c = ci[i], sn = si[i], d0 = h[i];
        h[i] = c * d0 + sn * h[i + 1];
        h[i + 1] = -sn * d0 + c * h[i + 1];
      }
      double r = 1.0 / sqrt(h[inner] * h[inner] + h[inner + 1] * h[inner + 1]);
      si[inner] = h[inner + 1] * r;
      ci[inner] = h[inner] * r;
      h[inner] = ci[inner] * h[inner] + si[inner] * h[inner + 1];
      gam[inner + 1] = -si[inner] * gam[inner];
      gam[inner] *= ci[inner];
      for (int i = 0; i < dimk; ++i) Hm[i * m + inner] = h[i];
      rho = fabs(gam[dimk]);
      if (history) history[acc] = rho;
      if (rho <= tol) state = 1;
      else if (acc >= max_it) state = 2;
    }
    /* back substitution H y = gamma, x += V y */
    double *y = (double *)calloc(dimk + 1, sizeof(double));
    for (int i = dimk - 1; i >= 0; --i) {
      double t = gam[i];
      for (int j = i + 1; j < dimk; ++j) t -= Hm[i * m + j] * y[j];
      y[i] = t / Hm[i * m + i];
    }
    for (int i = 0; i < dimk; ++i)
      for (long j = 0; j < N; ++j) x[j] += y[i] * V[i][j];
    free(y);
  } while (state == 0);
  for (int i = 0; i <= m; ++i) free(V[i]);
  free(V);
  free(p);
  free(Hm);
  free(h);
  free(gam);
  free(ci);
  free(si);
  return acc;
}
