// Host-side 1D finite-element data of degree k on the reference cell [0,1]
// (FP64), the vertex-patch matrices and their interior generalized
// eigendecomposition.  Replaces LevelVertexPatch::reinit_tensor_product
// (include/patch_base.template.cuh:709-1205) and TensorProductData
// (include/tensor_product.h:60-284) of the reference, without deal.II.
#pragma once

#include <vector>

namespace tps {

constexpr int kMaxDegree = 7;

struct DegreeData {
  int k = 0;                  // polynomial degree
  std::vector<double> nodes;  // k+1 Gauss-Lobatto support points on [0,1]
  std::vector<double> cmass;  // (k+1)^2 cell mass on [0,1], QGauss(k+1)
  std::vector<double> clap;   // (k+1)^2 cell stiffness on [0,1]
  std::vector<double> pmass;  // (2k+1)^2 vertex-patch mass (two reference cells)
  std::vector<double> plap;   // (2k+1)^2 vertex-patch stiffness
  // Interior generalized eigenpairs of the patch on REFERENCE cells:
  // plap_I v = mu pmass_I v, V^T pmass_I V = I, eigenvectors as columns
  // (evec[i*m + j] = v_j[i]), exactly even/odd under reflection.  Columns
  // 0..k-1 hold the k even modes, columns k..2k-2 the k-1 odd modes, each
  // group in ascending eigenvalue order.
  std::vector<double> evec;   // m^2, m = 2k-1
  std::vector<double> eval;   // m, ordered like the columns of evec
  std::vector<double> prol;   // (2k+1) x (k+1): coarse basis at child nodes
  // QGauss(k+1) on [0,1]: points, weights, and the basis at the points
  // (qshape[q * (k+1) + i] = phi_i(xq_q)), for right-hand-side assembly
  std::vector<double> qpoint, qweight, qshape;
};

// Builds every table above for degree k (1 <= k <= kMaxDegree).
DegreeData make_degree_data(int k);

// Inverse of the reference-cell interior patch matrix (the Exact local
// solver, include/loop_kernel.cuh:241-327): A_II = sum over the dim
// directions of the interior patch stiffness in that direction times the
// interior patch mass in the others, assembled densely (x fastest,
// (2k-1)^dim rows) and inverted by Cholesky factorisation in FP64.  Returns
// the full symmetric inverse, row-major.
std::vector<double> dense_patch_inverse(const DegreeData &D, int dim);

// B operand image of the 3D patch-GEMM smoother (smoother3d_gemm.cuh).  The
// patch step x_I = G u, G = [A_II^{-1} | -A_II^{-1} A_IB] over the (2k+1)^3
// box (reference-cell A, FP64), split by the parity of the box in z:
//   G_E (k (2k-1)^2 rows, (k+1)(2k+1)^2 columns), G_O ((k-1)(2k-1)^2 rows,
//   k (2k+1)^2 columns),
// row index zp * (2k-1)^2 + yi * (2k-1) + xi (zp: interior plane pair, k-1 the
// centre plane), column index p * (2k+1)^2 + y * (2k+1) + x (p: box plane
// pair, k the centre plane), the factors 1/2 of the folding included.  Each
// block is cut into chunks of `ck` columns; a chunk holds `nb` rows (zero
// padded) in the K-major no-swizzle operand layout of tcgen05 (8-row groups
// of ck/4 core matrices of 8 rows x 16 bytes), values rounded to nearest TF32.
// Returns G_E's chunks followed by G_O's as FP32 words.
std::vector<float> patch_gemm_image(const DegreeData &D, int nbe, int nbo, int ck);
// The same blocks with a choice of column order and precision: order 0 as
// above; order 1 lists, per box plane pair p, the entries x = 0..2k-1 of the
// rows y = 0..2k (column p (2k+1) 2k + y 2k + x) and after all plane pairs
// the x = 2k entries (column (pairs) (2k+1) 2k + p (2k+1) + y), so that a
// chunk of 3 * 2k columns is three box rows of one plane pair.  With split,
// a second image of the same size follows with the TF32 residuals
// tf32(v - tf32(v)) (the low parts of a three-product TF32 split).
std::vector<float> patch_gemm_image_ordered(const DegreeData &D, int nbe, int nbo, int ck, int order, bool split);

// Inverse of the symmetric positive definite n x n matrix A (row-major,
// overwritten): Cholesky factorisation A = L L^T, W = L^{-1}, A^{-1} = W^T W,
// every inner product over contiguous rows, independent rows on host threads
// (OpenMP).  Throws std::runtime_error if A is not positive definite.
std::vector<double> spd_inverse(std::vector<double> &A, int n);

// Symmetric-definite generalized eigenproblem A v = lambda B v (FP64,
// Cholesky + cyclic Jacobi); V column-major-as-rows like DegreeData::evec.
void generalized_eigen(int m, const double *A, const double *B, double *V, double *lambda);

}  // namespace tps
