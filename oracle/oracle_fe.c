/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle for the vertex-patch Schwarz MG path.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 * Parity status: UNPINNED against the reference. The reference
 * (LuciaZhang9/GPUTensorProductSmoother) needs deal.II >= 9.3 built with CUDA
 * and MPI (CMakeLists.txt:81-102), ships no golden vectors and has no
 * assertion-based tests; the oracle is instead pinned against independent
 * numpy/scipy fixtures under tests/golden/ and mathematical known answers.
 *
 * This file: 1D finite-element data on the reference cell [0,1] and the FP64
 * generalized symmetric eigensolver.
 *
 *  - FE_Q(k) / FE_DGQ(k) are Lagrange bases on the k+1 Gauss-Lobatto points
 *    (deal.II's default support points; used by the reference through
 *    FE_DGQ<1> in include/patch_base.template.cuh:713 and FE_Q<1> in
 *    include/tensor_product.h:67).
 *  - Quadrature is QGauss(k+1) (include/patch_base.template.cuh:717,
 *    include/tensor_product.h:88), exact for the mass and stiffness integrals.
 *  - The 1D cell mass/stiffness follow include/patch_base.template.cuh:727-762;
 *    the patch matrices (two overlapping cells) follow :749-788.
 *  - The interior generalized eigenproblem L v = lambda M v with V^T M V = I
 *    restates deal.II TensorProductMatrixSymmetricSum::reinit as called from
 *    include/tensor_product.h:208-210 (mass/derivative on the 2k-1 interior
 *    patch DoFs of a mesh with 2^level cells, tensor_product.h:60-106).
 *  - The 1D prolongation (coarse basis evaluated at the 2k+1 child nodes) is
 *    the matrix deal.II's internal::MGTransfer::setup_transfer builds for
 *    include/cuda_mg_transfer.template.cuh:490-502.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

/* Legendre P_n(x) and P_n'(x) on [-1,1] by the three-term recurrence. */
static void legendre(int n, double x, double *p, double *dp)
{
  double p0 = 1.0, p1 = x;
  if (n == 0) { *p = 1.0; *dp = 0.0; return; }
  for (int j = 1; j < n; ++j) {
    double p2 = ((2.0 * j + 1.0) * x * p1 - j * p0) / (j + 1.0);
    p0 = p1;
    p1 = p2;
  }
  *p = p1;
  /* derivative from (x^2-1) P_n' = n (x P_n - P_{n-1}); callers avoid |x|=1 */
  *dp = n * (x * p1 - p0) / (x * x - 1.0);
}

/* Gauss-Legendre points/weights mapped to [0,1]. */
void orc_gauss(int nq, double *x, double *w)
{
  for (int i = 0; i < nq; ++i) {
    double t = cos(M_PI * (i + 0.75) / (nq + 0.5));
    for (int it = 0; it < 100; ++it) {
      double p, dp;
      legendre(nq, t, &p, &dp);
      double dt = p / dp;
      t -= dt;
      if (fabs(dt) < 1e-16) break;
    }
    double p, dp;
    legendre(nq, t, &p, &dp);
    /* ascending order on [0,1] */
    x[nq - 1 - i] = 0.5 * (t + 1.0);
    w[nq - 1 - i] = 1.0 / ((1.0 - t * t) * dp * dp);
  }
}

/* k+1 Gauss-Lobatto points on [0,1]: 0, 1 and the roots of P_k'. */
void orc_gauss_lobatto(int k, double *x)
{
  x[0] = 0.0;
  x[k] = 1.0;
  for (int i = 1; i < k; ++i) {
    double t = -cos(M_PI * i / k);
    for (int it = 0; it < 100; ++it) {
      double p, dp;
      legendre(k, t, &p, &dp);
      /* P'' from the Legendre ODE (1-t^2)P'' - 2tP' + k(k+1)P = 0 */
      double d2p = (2.0 * t * dp - k * (k + 1.0) * p) / (1.0 - t * t);
      double dt = dp / d2p;
      t -= dt;
      if (fabs(dt) < 1e-16) break;
    }
    x[i] = 0.5 * (t + 1.0);
  }
}

static double lagrange_value(const double *nodes, int np, int i, double x)
{
  double v = 1.0;
  for (int m = 0; m < np; ++m)
    if (m != i) v *= (x - nodes[m]) / (nodes[i] - nodes[m]);
  return v;
}

static double lagrange_deriv(const double *nodes, int np, int i, double x)
{
  double s = 0.0;
  for (int m = 0; m < np; ++m) {
    if (m == i) continue;
    double t = 1.0 / (nodes[i] - nodes[m]);
    for (int l = 0; l < np; ++l)
      if (l != i && l != m) t *= (x - nodes[l]) / (nodes[i] - nodes[l]);
    s += t;
  }
  return s;
}

/*
 * 1D data of degree k on the reference cell [0,1]:
 *   nodes[k+1], mass[(k+1)^2], lap[(k+1)^2] (row-major, symmetric),
 *   prol[(2k+1)*(k+1)]: value of coarse basis c at fine node f of the two
 *   children [0,1/2], [1/2,1]; row f, column c.
 */
int orc_fe1d(int k, double *nodes, double *mass, double *lap, double *prol)
{
  if (k < 1 || k > ORC_MAXK) return -1;
  const int np = k + 1, nq = k + 1;
  double xq[ORC_MAXK + 1], wq[ORC_MAXK + 1];
  double gl[ORC_MAXK + 1];
  orc_gauss(nq, xq, wq);
  orc_gauss_lobatto(k, gl);
  if (nodes) memcpy(nodes, gl, sizeof(double) * np);
  for (int i = 0; i < np; ++i)
    for (int j = 0; j < np; ++j) {
      double sm = 0.0, sl = 0.0;
      for (int q = 0; q < nq; ++q) {
        sm += lagrange_value(gl, np, i, xq[q]) * lagrange_value(gl, np, j, xq[q]) * wq[q];
        sl += lagrange_deriv(gl, np, i, xq[q]) * lagrange_deriv(gl, np, j, xq[q]) * wq[q];
      }
      if (mass) mass[i * np + j] = sm;
      if (lap) lap[i * np + j] = sl;
    }
  if (prol) {
    const int nf = 2 * k + 1;
    for (int f = 0; f < nf; ++f) {
      double x = (f <= k) ? 0.5 * gl[f] : 0.5 + 0.5 * gl[f - k];
      for (int c = 0; c < np; ++c) {
        double v = lagrange_value(gl, np, c, x);
        /* exact interpolation at coinciding nodes */
        if (fabs(v) < 1e-15) v = 0.0;
        if (fabs(v - 1.0) < 1e-15) v = 1.0;
        prol[f * np + c] = v;
      }
    }
  }
  return 0;
}

/*
 * Patch (2k+1)^2 matrices on reference cells: the two cells' matrices summed
 * with an overlap at the shared vertex (include/patch_base.template.cuh:749-788).
 */
int orc_patch_matrices(int k, double *pmass, double *plap)
{
  if (k < 1 || k > ORC_MAXK) return -1;
  const int np = k + 1, n1 = 2 * k + 1;
  double mass[(ORC_MAXK + 1) * (ORC_MAXK + 1)], lap[(ORC_MAXK + 1) * (ORC_MAXK + 1)];
  orc_fe1d(k, NULL, mass, lap, NULL);
  memset(pmass, 0, sizeof(double) * n1 * n1);
  memset(plap, 0, sizeof(double) * n1 * n1);
  for (int i = 0; i < np; ++i)
    for (int j = 0; j < np; ++j) {
      pmass[i * n1 + j] += mass[i * np + j];
      pmass[(i + k) * n1 + (j + k)] += mass[i * np + j];
      plap[i * n1 + j] += lap[i * np + j];
      plap[(i + k) * n1 + (j + k)] += lap[i * np + j];
    }
  return 0;
}

/* Cyclic Jacobi eigen-decomposition of a symmetric m x m matrix A (destroyed).
 * On return Q holds eigenvectors as columns and d the eigenvalues. */
static void jacobi_eig(int m, double *A, double *Q, double *d)
{
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j) Q[i * m + j] = (i == j);
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) {
        tot += A[i * m + j] * A[i * m + j];
        if (i != j) off += A[i * m + j] * A[i * m + j];
      }
    if (off <= 1e-32 * tot) break;
    for (int p = 0; p < m - 1; ++p)
      for (int q = p + 1; q < m; ++q) {
        double apq = A[p * m + q];
        if (fabs(apq) < 1e-300) continue;
        double theta = (A[q * m + q] - A[p * m + p]) / (2.0 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int r = 0; r < m; ++r) {
          double arp = A[r * m + p], arq = A[r * m + q];
          A[r * m + p] = c * arp - s * arq;
          A[r * m + q] = s * arp + c * arq;
        }
        for (int r = 0; r < m; ++r) {
          double apr = A[p * m + r], aqr = A[q * m + r];
          A[p * m + r] = c * apr - s * aqr;
          A[q * m + r] = s * apr + c * aqr;
        }
        for (int r = 0; r < m; ++r) {
          double qrp = Q[r * m + p], qrq = Q[r * m + q];
          Q[r * m + p] = c * qrp - s * qrq;
          Q[r * m + q] = s * qrp + c * qrq;
        }
      }
  }
  for (int i = 0; i < m; ++i) d[i] = A[i * m + i];
}

/*
 * Generalized symmetric-definite eigenproblem L v = lambda M v (FP64):
 * Cholesky M = C C^T, Jacobi on C^{-1} L C^{-T}, V = C^{-T} Q, so that
 * V^T M V = I and V^T L V = diag(lambda).  Eigenvalues ascending.
 * V is returned row-major with eigenvectors as COLUMNS: V[i*m+j] = v_j[i].
 */
int orc_gen_eig(int m, const double *L, const double *M, double *V, double *lam)
{
  if (m < 1 || m > 2 * ORC_MAXK + 1) return -1;
  double C[ORC_MAXN1 * ORC_MAXN1], K[ORC_MAXN1 * ORC_MAXN1], T[ORC_MAXN1 * ORC_MAXN1];
  double Q[ORC_MAXN1 * ORC_MAXN1], d[ORC_MAXN1];
  memset(C, 0, sizeof(C));
  for (int j = 0; j < m; ++j) {
    double s = M[j * m + j];
    for (int p = 0; p < j; ++p) s -= C[j * m + p] * C[j * m + p];
    if (s <= 0) return -2;
    C[j * m + j] = sqrt(s);
    for (int i = j + 1; i < m; ++i) {
      double t = M[i * m + j];
      for (int p = 0; p < j; ++p) t -= C[i * m + p] * C[j * m + p];
      C[i * m + j] = t / C[j * m + j];
    }
  }
  /* T = C^{-1} L  (forward substitution per column) */
  for (int c = 0; c < m; ++c)
    for (int i = 0; i < m; ++i) {
      double t = L[i * m + c];
      for (int p = 0; p < i; ++p) t -= C[i * m + p] * T[p * m + c];
      T[i * m + c] = t / C[i * m + i];
    }
  /* K = T C^{-T} = (C^{-1} T^T)^T ; solve C Y = T^T, K = Y^T */
  for (int c = 0; c < m; ++c)
    for (int i = 0; i < m; ++i) {
      double t = T[c * m + i];
      for (int p = 0; p < i; ++p) t -= C[i * m + p] * K[c * m + p];
      K[c * m + i] = t / C[i * m + i];
    }
  /* symmetrize against rounding */
  for (int i = 0; i < m; ++i)
    for (int j = i + 1; j < m; ++j) {
      double a = 0.5 * (K[i * m + j] + K[j * m + i]);
      K[i * m + j] = K[j * m + i] = a;
    }
  jacobi_eig(m, K, Q, d);
  /* V = C^{-T} Q : back substitution C^T V = Q */
  for (int c = 0; c < m; ++c)
    for (int i = m - 1; i >= 0; --i) {
      double t = Q[i * m + c];
      for (int p = i + 1; p < m; ++p) t -= C[p * m + i] * V[p * m + c];
      V[i * m + c] = t / C[i * m + i];
    }
  /* sort ascending */
  for (int a = 0; a < m; ++a) {
    int best = a;
    for (int b = a + 1; b < m; ++b)
      if (d[b] < d[best]) best = b;
    if (best != a) {
      double t = d[a];
      d[a] = d[best];
      d[best] = t;
      for (int i = 0; i < m; ++i) {
        double v = V[i * m + a];
        V[i * m + a] = V[i * m + best];
        V[i * m + best] = v;
      }
    }
  }
  memcpy(lam, d, sizeof(double) * m);
  return 0;
}

/*
 * Physical interior eigenpairs of a vertex patch of a uniform mesh with cell
 * size h: M_I = h * Mpatch[1..m], L_I = Lpatch[1..m] / h, m = 2k-1.
 * (include/tensor_product.h:112-210 restricted to the interior DoFs.)
 */
int orc_patch_eigen(int k, double h, double *S, double *lam)
{
  const int n1 = 2 * k + 1, m = 2 * k - 1;
  double pm[ORC_MAXN1 * ORC_MAXN1], pl[ORC_MAXN1 * ORC_MAXN1];
  double MI[ORC_MAXN1 * ORC_MAXN1], LI[ORC_MAXN1 * ORC_MAXN1];
  if (orc_patch_matrices(k, pm, pl)) return -1;
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j) {
      MI[i * m + j] = h * pm[(i + 1) * n1 + (j + 1)];
      LI[i * m + j] = pl[(i + 1) * n1 + (j + 1)] / h;
    }
  return orc_gen_eig(m, LI, MI, S, lam);
}
