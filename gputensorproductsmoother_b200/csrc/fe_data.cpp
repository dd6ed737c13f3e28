// Host 1D finite-element data and the FP64 generalized eigensolver.
//
// Restates, without deal.II, what the reference obtains from FE_DGQ<1>/FE_Q<1>
// + QGauss<1>(k+1) (include/patch_base.template.cuh:713-762,
// include/tensor_product.h:112-189) and from
// TensorProductMatrixSymmetricSum::reinit (include/tensor_product.h:208-210).
// The eigendecomposition runs in FP64 on the host (the reference runs it in
// the V-cycle precision, include/patch_base.template.cuh:791-806) and splits
// the centro-symmetric interior problem into its even and odd halves so the
// eigenvectors are exactly symmetric / antisymmetric, which the kernels use
// to halve the fast-diagonalization work.
#include "fe_data.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>

namespace tps {
namespace {

// Legendre polynomial value and first two derivatives on [-1,1].
void legendre_eval(int n, double t, double &p, double &dp)
{
  double pm1 = 1.0, pn = t;
  if (n == 0) {
    p = 1.0;
    dp = 0.0;
    return;
  }
  for (int j = 2; j <= n; ++j) {
    const double pj = ((2.0 * j - 1.0) * t * pn - (j - 1.0) * pm1) / j;
    pm1 = pn;
    pn = pj;
  }
  p = pn;
  dp = n * (pm1 - t * pn) / (1.0 - t * t);
}

std::vector<double> gauss_lobatto(int k)
{
  std::vector<double> x(k + 1);
  x[0] = 0.0;
  x[k] = 1.0;
  for (int i = 1; i < k; ++i) {
    double t = -std::cos(M_PI * i / k);
    for (int it = 0; it < 200; ++it) {
      double p, dp;
      legendre_eval(k, t, p, dp);
      const double d2p = (2.0 * t * dp - k * (k + 1.0) * p) / (1.0 - t * t);
      const double step = dp / d2p;
      t -= step;
      if (std::fabs(step) < 1e-17) break;
    }
    x[i] = 0.5 * (1.0 + t);
  }
  return x;
}

void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w)
{
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < n; ++i) {
    double t = -std::cos(M_PI * (i + 0.75) / (n + 0.5));
    for (int it = 0; it < 200; ++it) {
      double p, dp;
      legendre_eval(n, t, p, dp);
      const double step = p / dp;
      t -= step;
      if (std::fabs(step) < 1e-17) break;
    }
    double p, dp;
    legendre_eval(n, t, p, dp);
    x[i] = 0.5 * (1.0 + t);
    w[i] = 1.0 / ((1.0 - t * t) * dp * dp);
  }
}

// Lagrange basis on `nodes`: value and derivative of basis i at x.
void lagrange(const std::vector<double> &nodes, int i, double x, double &v, double &d)
{
  const int np = static_cast<int>(nodes.size());
  v = 1.0;
  d = 0.0;
  for (int m = 0; m < np; ++m) {
    if (m == i) continue;
    const double inv = 1.0 / (nodes[i] - nodes[m]);
    d = d * (x - nodes[m]) * inv + v * inv;  // product rule, accumulated
    v *= (x - nodes[m]) * inv;
  }
}

void cholesky_lower(int m, std::vector<double> &C, const double *B)
{
  C.assign(m * m, 0.0);
  for (int j = 0; j < m; ++j) {
    double s = B[j * m + j];
    for (int p = 0; p < j; ++p) s -= C[j * m + p] * C[j * m + p];
    if (!(s > 0)) throw std::runtime_error("mass matrix not positive definite");
    C[j * m + j] = std::sqrt(s);
    for (int i = j + 1; i < m; ++i) {
      double t = B[i * m + j];
      for (int p = 0; p < j; ++p) t -= C[i * m + p] * C[j * m + p];
      C[i * m + j] = t / C[j * m + j];
    }
  }
}

// Symmetric Jacobi; A destroyed, Q eigenvectors as columns.
void jacobi(int m, std::vector<double> &A, std::vector<double> &Q, std::vector<double> &d)
{
  Q.assign(m * m, 0.0);
  for (int i = 0; i < m; ++i) Q[i * m + i] = 1.0;
  for (int sweep = 0; sweep < 64; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) (i == j ? diag : off) += A[i * m + j] * A[i * m + j];
    if (off <= 1e-34 * (diag + off)) break;
    for (int p = 0; p < m; ++p)
      for (int q = p + 1; q < m; ++q) {
        const double apq = A[p * m + q];
        if (apq == 0.0) continue;
        const double tau = (A[q * m + q] - A[p * m + p]) / (2.0 * apq);
        const double t = std::copysign(1.0, tau) / (std::fabs(tau) + std::hypot(1.0, tau));
        const double c = 1.0 / std::hypot(1.0, t), s = t * c;
        for (int r = 0; r < m; ++r) {
          const double a = A[r * m + p], b = A[r * m + q];
          A[r * m + p] = c * a - s * b;
          A[r * m + q] = s * a + c * b;
        }
        for (int r = 0; r < m; ++r) {
          const double a = A[p * m + r], b = A[q * m + r];
          A[p * m + r] = c * a - s * b;
          A[q * m + r] = s * a + c * b;
        }
        for (int r = 0; r < m; ++r) {
          const double a = Q[r * m + p], b = Q[r * m + q];
          Q[r * m + p] = c * a - s * b;
          Q[r * m + q] = s * a + c * b;
        }
      }
  }
  d.resize(m);
  for (int i = 0; i < m; ++i) d[i] = A[i * m + i];
}

}  // namespace

void generalized_eigen(int m, const double *A, const double *B, double *V, double *lambda)
{
  std::vector<double> C, W(m * m), K(m * m), Q, d;
  cholesky_lower(m, C, B);
  // W = C^{-1} A
  for (int col = 0; col < m; ++col)
    for (int i = 0; i < m; ++i) {
      double t = A[i * m + col];
      for (int p = 0; p < i; ++p) t -= C[i * m + p] * W[p * m + col];
      W[i * m + col] = t / C[i * m + i];
    }
  // K = W C^{-T}: row r of K solves C k_r = w_r (W symmetric-congruent)
  for (int r = 0; r < m; ++r)
    for (int i = 0; i < m; ++i) {
      double t = W[r * m + i];
      for (int p = 0; p < i; ++p) t -= C[i * m + p] * K[r * m + p];
      K[r * m + i] = t / C[i * m + i];
    }
  for (int i = 0; i < m; ++i)
    for (int j = i + 1; j < m; ++j) K[i * m + j] = K[j * m + i] = 0.5 * (K[i * m + j] + K[j * m + i]);
  jacobi(m, K, Q, d);
  // V = C^{-T} Q
  std::vector<double> Vt(m * m);
  for (int col = 0; col < m; ++col)
    for (int i = m - 1; i >= 0; --i) {
      double t = Q[i * m + col];
      for (int p = i + 1; p < m; ++p) t -= C[p * m + i] * Vt[p * m + col];
      Vt[i * m + col] = t / C[i * m + i];
    }
  std::vector<int> order(m);
  for (int i = 0; i < m; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](int a, int b) { return d[a] < d[b]; });
  for (int j = 0; j < m; ++j) {
    lambda[j] = d[order[j]];
    for (int i = 0; i < m; ++i) V[i * m + j] = Vt[i * m + order[j]];
  }
}

DegreeData make_degree_data(int k)
{
  if (k < 1 || k > kMaxDegree) throw std::runtime_error("degree out of range");
  DegreeData D;
  D.k = k;
  const int np = k + 1, n1 = 2 * k + 1, m = 2 * k - 1;
  D.nodes = gauss_lobatto(k);
  std::vector<double> xq, wq;
  gauss_legendre(k + 1, xq, wq);
  D.cmass.assign(np * np, 0.0);
  D.clap.assign(np * np, 0.0);
  D.qpoint = xq;
  D.qweight = wq;
  D.qshape.assign(np * np, 0.0);
  for (int q = 0; q < k + 1; ++q) {
    std::vector<double> v(np), dv(np);
    for (int i = 0; i < np; ++i) lagrange(D.nodes, i, xq[q], v[i], dv[i]);
    for (int i = 0; i < np; ++i) D.qshape[q * np + i] = v[i];
    for (int i = 0; i < np; ++i)
      for (int j = 0; j < np; ++j) {
        D.cmass[i * np + j] += wq[q] * v[i] * v[j];
        D.clap[i * np + j] += wq[q] * dv[i] * dv[j];
      }
  }
  D.pmass.assign(n1 * n1, 0.0);
  D.plap.assign(n1 * n1, 0.0);
  for (int cell = 0; cell < 2; ++cell)
    for (int i = 0; i < np; ++i)
      for (int j = 0; j < np; ++j) {
        D.pmass[(i + cell * k) * n1 + j + cell * k] += D.cmass[i * np + j];
        D.plap[(i + cell * k) * n1 + j + cell * k] += D.clap[i * np + j];
      }
  // interior blocks, then even/odd split around the centre DoF c = k-1
  std::vector<double> MI(m * m), LI(m * m);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j) {
      MI[i * m + j] = D.pmass[(i + 1) * n1 + j + 1];
      LI[i * m + j] = D.plap[(i + 1) * n1 + j + 1];
    }
  const int c = k - 1;  // centre index of the interior
  const double r2 = std::sqrt(0.5);
  // even basis: (e_i + e_{m-1-i})/sqrt2 for i < c, and e_c ; odd: (e_i - e_{m-1-i})/sqrt2
  const int ne = c + 1, no = c;
  std::vector<double> Qe(m * ne, 0.0), Qo(m * std::max(no, 1), 0.0);
  for (int i = 0; i < c; ++i) {
    Qe[i * ne + i] = r2;
    Qe[(m - 1 - i) * ne + i] = r2;
    Qo[i * no + i] = r2;
    Qo[(m - 1 - i) * no + i] = -r2;
  }
  Qe[c * ne + c] = 1.0;
  auto project = [&](const std::vector<double> &Qx, int nx, const std::vector<double> &A) {
    std::vector<double> R(nx * nx, 0.0);
    for (int a = 0; a < nx; ++a)
      for (int b = 0; b < nx; ++b) {
        double s = 0.0;
        for (int i = 0; i < m; ++i)
          for (int j = 0; j < m; ++j) s += Qx[i * nx + a] * A[i * m + j] * Qx[j * nx + b];
        R[a * nx + b] = s;
      }
    return R;
  };
  // Mode order: the C+1 reflection-even eigenvectors first (ascending), then
  // the C odd ones (ascending).  The kernels rely on this order to apply S and
  // S^T on folded half-lines with compile-time parity.
  D.evec.assign(m * m, 0.0);
  D.eval.assign(m, 0.0);
  int col = 0;
  for (int part = 0; part < 2; ++part) {
    const int nx = part == 0 ? ne : no;
    if (nx == 0) continue;
    const std::vector<double> &Qx = part == 0 ? Qe : Qo;
    std::vector<double> Ms = project(Qx, nx, MI), Ls = project(Qx, nx, LI);
    std::vector<double> W(nx * nx), lam(nx);
    generalized_eigen(nx, Ls.data(), Ms.data(), W.data(), lam.data());
    for (int j = 0; j < nx; ++j, ++col) {
      std::vector<double> v(m, 0.0);
      for (int i = 0; i < m; ++i)
        for (int a = 0; a < nx; ++a) v[i] += Qx[i * nx + a] * W[a * nx + j];
      // make the reflection symmetry exact
      for (int i = 0; i < c; ++i) {
        const double s = part == 0 ? 0.5 * (v[i] + v[m - 1 - i]) : 0.5 * (v[i] - v[m - 1 - i]);
        v[i] = s;
        v[m - 1 - i] = part == 0 ? s : -s;
      }
      if (part == 1) v[c] = 0.0;
      D.eval[col] = lam[j];
      for (int i = 0; i < m; ++i) D.evec[i * m + col] = v[i];
    }
  }
  // 1D prolongation: coarse basis evaluated at the child nodes
  D.prol.assign(n1 * np, 0.0);
  for (int f = 0; f < n1; ++f) {
    const double x = f <= k ? 0.5 * D.nodes[f] : 0.5 + 0.5 * D.nodes[f - k];
    for (int cc = 0; cc < np; ++cc) {
      double v, d;
      lagrange(D.nodes, cc, x, v, d);
      if (std::fabs(v) < 1e-14) v = 0.0;
      if (std::fabs(v - 1.0) < 1e-14) v = 1.0;
      D.prol[f * np + cc] = v;
    }
  }
  return D;
}

std::vector<double> dense_patch_inverse(const DegreeData &D, int dim)
{
  const int k = D.k, n1 = 2 * k + 1, m = 2 * k - 1;
  int n = 1;
  for (int d = 0; d < dim; ++d) n *= m;
  auto Mi = [&](int i, int j) { return D.pmass[(i + 1) * n1 + j + 1]; };
  auto Li = [&](int i, int j) { return D.plap[(i + 1) * n1 + j + 1]; };
  const size_t nn = static_cast<size_t>(n);
  std::vector<double> A(nn * nn);
  for (int e = 0; e < n; ++e) {
    const int ex = e % m, ey = (e / m) % m, ez = dim == 3 ? e / (m * m) : 0;
    for (int f = 0; f < n; ++f) {
      const int fx = f % m, fy = (f / m) % m, fz = dim == 3 ? f / (m * m) : 0;
      double v;
      if (dim == 3)
        v = Li(ex, fx) * Mi(ey, fy) * Mi(ez, fz) + Mi(ex, fx) * Li(ey, fy) * Mi(ez, fz) +
            Mi(ex, fx) * Mi(ey, fy) * Li(ez, fz);
      else
        v = Li(ex, fx) * Mi(ey, fy) + Mi(ex, fx) * Li(ey, fy);
      A[e * nn + f] = v;
    }
  }
  return spd_inverse(A, n);
}

namespace {
// round to the nearest TF32 value, ties away from zero (as cvt.rna.tf32.f32)
float round_tf32(double v)
{
  float f = static_cast<float>(v);
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u = (u + 0x1000u) & 0xFFFFE000u;
  std::memcpy(&f, &u, 4);
  return f;
}
}  // namespace

std::vector<float> patch_gemm_image(const DegreeData &D, int nbe, int nbo, int ck)
{
  return patch_gemm_image_ordered(D, nbe, nbo, ck, 0, false);
}

std::vector<float> patch_gemm_image_ordered(const DegreeData &D, int nbe, int nbo, int ck, int order, bool split)
{
  const int k = D.k, n1 = 2 * k + 1, m = 2 * k - 1;
  const int nb = n1 * n1 * n1, ni = m * m * m, pl = n1 * n1, ipl = m * m;
  const std::vector<double> inv = dense_patch_inverse(D, 3);  // ni x ni
  auto idx_box = [&](int z, int y, int x) { return x + n1 * (y + n1 * z); };
  // G (ni x nb): interior columns A_II^{-1}, ring columns -A_II^{-1} A_IB
  std::vector<double> G(static_cast<size_t>(ni) * nb, 0.0);
  std::vector<double> aib(static_cast<size_t>(ni) * nb, 0.0);  // A(i, q) for ring q
  const double *Mm = D.pmass.data(), *Ll = D.plap.data();
  for (int i = 0; i < ni; ++i) {
    const int ix = 1 + i % m, iy = 1 + (i / m) % m, iz = 1 + i / (m * m);
    for (int q = 0; q < nb; ++q) {
      const int qx = q % n1, qy = (q / n1) % n1, qz = q / pl;
      const bool ring = qx == 0 || qx == n1 - 1 || qy == 0 || qy == n1 - 1 || qz == 0 || qz == n1 - 1;
      if (!ring) continue;
      aib[static_cast<size_t>(i) * nb + q] =
          Ll[ix * n1 + qx] * Mm[iy * n1 + qy] * Mm[iz * n1 + qz] + Mm[ix * n1 + qx] * Ll[iy * n1 + qy] * Mm[iz * n1 + qz] +
          Mm[ix * n1 + qx] * Mm[iy * n1 + qy] * Ll[iz * n1 + qz];
    }
  }
  for (int i = 0; i < ni; ++i) {
    double *g = &G[static_cast<size_t>(i) * nb];
    for (int j = 0; j < ni; ++j) {
      const double w = inv[static_cast<size_t>(i) * ni + j];
      const int jx = 1 + j % m, jy = 1 + (j / m) % m, jz = 1 + j / (m * m);
      g[idx_box(jz, jy, jx)] += w;
      const double *a = &aib[static_cast<size_t>(j) * nb];
      for (int q = 0; q < nb; ++q) g[q] -= w * a[q];
    }
  }
  // z-parity blocks
  auto grow = [&](int zi, int r) { return &G[static_cast<size_t>(zi * ipl + r) * nb]; };
  const int ne = k * ipl, no = (k - 1) * ipl, ke = (k + 1) * pl, ko = k * pl;
  auto coef = [&](bool odd_out, bool odd_in, int zp, int r, int p, int s) {
    // output side: E = (y(zp) + y(m-1-zp)) / 2 (zp < k-1), y(k-1) for the centre;
    // O = (y(zp) - y(m-1-zp)) / 2.  Input side: e_p <- (G(p) + G(n1-1-p)) / 2
    // (p < k), G(k) for the centre; o_p <- (G(p) - G(n1-1-p)) / 2.
    auto in = [&](const double *row) {
      if (p == k) return row[p * pl + s];
      const double a = row[p * pl + s], b = row[(n1 - 1 - p) * pl + s];
      return odd_in ? 0.5 * (a - b) : 0.5 * (a + b);
    };
    if (zp == k - 1) return in(grow(zp, r));
    const double a = in(grow(zp, r)), b = in(grow(m - 1 - zp, r));
    return odd_out ? 0.5 * (a - b) : 0.5 * (a + b);
  };
  // K (column) order: 0 = p * (2k+1)^2 + s; 1 = the entries x < 2k of the box
  // rows first (p * (2k+1) * 2k + y * 2k + x), then the x = 2k entries
  // (rows_total + p * (2k+1) + y).  Returns false for a padding column.
  const int rw = n1 - 1, rpp = n1 * rw;
  auto colmap = [&](int col, int n_pp, int &p, int &s) {
    if (order == 0) {
      if (col >= n_pp * pl) return false;
      p = col / pl;
      s = col % pl;
      return true;
    }
    if (col < n_pp * rpp) {
      p = col / rpp;
      const int r = col % rpp;
      s = (r / rw) * n1 + r % rw;
      return true;
    }
    const int c2 = col - n_pp * rpp;
    if (c2 >= n_pp * n1) return false;
    p = c2 / n1;
    s = (c2 % n1) * n1 + rw;
    return true;
  };
  const int ke_cols = (k + 1) * pl, ko_cols = k * pl;
  const int ce = (ke_cols + ck - 1) / ck, co = (ko_cols + ck - 1) / ck;
  const size_t chunk_e = static_cast<size_t>(nbe) * ck, chunk_o = static_cast<size_t>(nbo) * ck;
  const size_t one = ce * chunk_e + co * chunk_o;
  std::vector<float> img((split ? 2 : 1) * one, 0.f);
  auto put = [&](float *base, int n, int kk, double v) {
    // K-major, no swizzle: 8-row groups of ck/4 core matrices (8 rows x 16 bytes);
    // with split, the TF32 residual v - tf32(v) goes to the second image
    const size_t at = ((n >> 3) * (ck / 4) * 128 + (n & 7) * 16 + (kk >> 2) * 128 + (kk & 3) * 4) / 4;
    const float hi = round_tf32(v);
    base[at] = hi;
    if (split) base[one + at] = round_tf32(v - static_cast<double>(hi));
  };
  for (int c = 0; c < ce; ++c)
    for (int n = 0; n < ne; ++n)
      for (int kk = 0; kk < ck; ++kk) {
        int p = 0, s = 0;
        if (!colmap(c * ck + kk, k + 1, p, s)) continue;
        const int zp = n / ipl, r = n % ipl;
        put(&img[c * chunk_e], n, kk, coef(false, false, zp, r, p, s));
      }
  float *go = img.data() + ce * chunk_e;
  for (int c = 0; c < co; ++c)
    for (int n = 0; n < no; ++n)
      for (int kk = 0; kk < ck; ++kk) {
        int p = 0, s = 0;
        if (!colmap(c * ck + kk, k, p, s)) continue;
        const int zp = n / ipl, r = n % ipl;
        put(go + c * chunk_o, n, kk, coef(true, true, zp, r, p, s));
      }
  return img;
}

std::vector<double> spd_inverse(std::vector<double> &A, int n)
{
  const size_t nn = static_cast<size_t>(n);
  // A = L L^T in the lower triangle: row j, then the rows below it in parallel
  for (size_t j = 0; j < nn; ++j) {
    double s = A[j * nn + j];
    for (size_t p = 0; p < j; ++p) s -= A[j * nn + p] * A[j * nn + p];
    if (!(s > 0.0)) throw std::runtime_error("matrix is not positive definite");
    const double d = std::sqrt(s);
    A[j * nn + j] = d;
    const double *lj = &A[j * nn];
#pragma omp parallel for schedule(static) if (nn - j > 256)
    for (long long i = static_cast<long long>(j) + 1; i < static_cast<long long>(nn); ++i) {
      double *li = &A[static_cast<size_t>(i) * nn];
      double t = li[j];
      for (size_t p = 0; p < j; ++p) t -= li[p] * lj[p];
      li[j] = t / d;
    }
  }
  // WT[c][p] = (L^{-1})[p][c] for p >= c; columns are independent
  std::vector<double> WT(nn * nn, 0.0);
#pragma omp parallel for schedule(dynamic, 8)
  for (long long cc = 0; cc < static_cast<long long>(nn); ++cc) {
    const size_t c = static_cast<size_t>(cc);
    double *w = &WT[c * nn];
    w[c] = 1.0 / A[c * nn + c];
    for (size_t i = c + 1; i < nn; ++i) {
      const double *li = &A[i * nn];
      double t = 0.0;
      for (size_t p = c; p < i; ++p) t += li[p] * w[p];
      w[i] = -t / li[i];
    }
  }
  // A^{-1}[i][j] = sum over p >= max(i, j) of W[p][i] W[p][j]
  std::vector<double> inv(nn * nn);
#pragma omp parallel for schedule(dynamic, 8)
  for (long long ii = 0; ii < static_cast<long long>(nn); ++ii) {
    const size_t i = static_cast<size_t>(ii);
    const double *wi = &WT[i * nn];
    for (size_t j = i; j < nn; ++j) {
      const double *wj = &WT[j * nn];
      double t = 0.0;
      for (size_t p = j; p < nn; ++p) t += wi[p] * wj[p];
      inv[i * nn + j] = t;
      inv[j * nn + i] = t;
    }
  }
  return inv;
}

}  // namespace tps
