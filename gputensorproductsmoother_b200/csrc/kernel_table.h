// Host-visible launch table: one instance per compiled degree k, defined in
// deg<k>.cu.  Entries are indexed [dim - 2][dtype] with dtype 0 = FP64,
// 1 = FP32.  No torch or deal.II types cross this boundary.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "fe_data.h"

namespace tps {

struct LevelGeomH {
  int n;      // cells per direction
  int N1;     // DoFs per direction
  int64_t N;  // DoFs
  double h;   // cell size
};

// Layout of a level vector: x fastest, row pitch sy >= N1, plane pitch sz
// (lexicographic: sy = N1, sz = N1^2; V-cycle work vectors pad sy to 16 bytes).
struct VecLayout {
  int N1;
  int64_t sy, sz;
};

// Opaque storage of the two TMA descriptors (CUtensorMap, 128 bytes each)
// of one smoother launch: x (patch boxes) and b (patch interiors).
struct SmootherMaps {
  alignas(64) unsigned char x[128];
  alignas(64) unsigned char b[128];
  int valid = 0;
  // views for the tensor-core smoother (FP32): the x box in its K-major
  // operand layout (rank 4) and the b interior (rank 3)
  alignas(64) unsigned char tx[128];
  alignas(64) unsigned char tb[128];
  int tc_valid = 0;
};

// compiled variants of the 3D smoother: patches per CTA batch default, half,
// quarter, one warp per patch, and two patches per warp (packed FP32)
constexpr int kSmootherVariants = 5;

struct KernelTable {
  int degree;
  // copy the 1D tables of this degree into constant memory of the current device
  cudaError_t (*upload)(const DegreeData &);
  // dst = A src on interior rows (mode 0) or dst = rhs - A src (mode 1);
  // boundary rows of dst are not written; layers (3D): cell layers per CTA
  // of the z-marching kernel, 1, 2, 4 or 8, or 0 for the default rule
  cudaError_t (*laplace[2][2])(const LevelGeomH &, const VecLayout &, void *dst, const void *src,
                               const void *rhs, int mode, int layers, cudaStream_t);
  // one colour of the patch sweep; maps (3D, TMA path) may be null; zero_x
  // declares x == 0 on entry; variant selects the 3D kernel shape
  // (0 default, 1 half, 2 quarter batch, 3 one warp per patch; see
  // smoother_ppb); err receives 1 if a
  // bounded wait gave up
  cudaError_t (*smoother[2][2])(const LevelGeomH &, const VecLayout &, void *x, const void *b,
                                int colour, double omega, int zero_x, int variant,
                                const SmootherMaps *maps, int *err, cudaStream_t);
  // TMA descriptors of the 3D smoother for vectors x, b with layout l ([dtype])
  cudaError_t (*encode_maps[2])(const VecLayout &l, void *x, const void *b, SmootherMaps *out);
  // fine += P coarse (interior fine DoFs); geometry of the COARSE level
  cudaError_t (*prolong[2][2])(const LevelGeomH &coarse, const VecLayout &lc, const VecLayout &lf,
                               void *fine, const void *coarse_v, void *tmp, cudaStream_t);
  // coarse (+)= R fine on interior coarse DoFs; geometry of the COARSE level
  cudaError_t (*restrict_[2][2])(const LevelGeomH &coarse, const VecLayout &lc,
                                 const VecLayout &lf, void *coarse_v, const void *fine, void *tmp,
                                 int add, cudaStream_t);
  // variable coefficient (kappa per cell, lexicographic cells, precision of the vector):
  // dst = A(kappa) src on interior rows (mode 0) or rhs - A(kappa) src (mode 1)
  cudaError_t (*kappa_laplace[2][2])(const LevelGeomH &, const VecLayout &, void *dst,
                                     const void *src, const void *rhs, const void *kappa, int mode,
                                     cudaStream_t);
  // one colour of the kappa patch sweep
  cudaError_t (*kappa_smoother[2][2])(const LevelGeomH &, const VecLayout &, void *x, const void *b,
                                      const void *kappa, int colour, double omega, cudaStream_t);
  // dst = M src (all rows, FP64) and e_c = lambda_c^T A_cell u_c (FP64)
  cudaError_t (*mass[2])(const LevelGeomH &, const VecLayout &, double *dst, const double *src,
                         cudaStream_t);
  cudaError_t (*cell_energy[2])(const LevelGeomH &, const VecLayout &, double *e, const double *u,
                                const double *lam, cudaStream_t);
  // b = sum over cells and QGauss(k+1) points of f phi_i JxW, interior rows
  // (FP64; f at the cells' Gauss points, cells then points lexicographic)
  cudaError_t (*assemble_rhs[2])(const LevelGeomH &, const VecLayout &, double *b, const double *fq, cudaStream_t);
  // 3D FP64 q = A p (z-marching kernel) with the p.q partial sums of a CG step
  // fused: one per CTA into partial (at most capacity), *ctas = their count
  cudaError_t (*laplace3d_dot)(const LevelGeomH &, const VecLayout &, void *dst, const void *src,
                               double *partial, int capacity, int layers, int *ctas, cudaStream_t);
  // the most CTAs laplace3d_dot launches on a level of n cells
  int (*laplace3d_ctas)(int n);
  // 3D colour step on the tensor cores (FP32 vectors, TF32 operands, FP32
  // accumulation; passes 3: three-term TF32 split, degree 4 only); null for
  // degree 1; needs maps->tc_valid
  cudaError_t (*smoother_tc)(const LevelGeomH &, const VecLayout &, void *x, const void *b, int colour,
                             double omega, int zero_x, const SmootherMaps *maps, int passes, int *err,
                             cudaStream_t);
  // the rank-4 TMA views of FP32 x and b (sets tc_valid when the layout allows them)
  cudaError_t (*encode_tc_maps)(const VecLayout &l, void *x, const void *b, SmootherMaps *out);
  // patches per CTA batch of smoother variant v (dtype 0 FP64, 1 FP32; 0 in
  // 2D; -1 for the one-warp-per-patch kernel)
  int (*smoother_ppb)(int dim, int dtype, int variant);
  // FP64 fine += P coarse with the coarse boundary values used ([dim - 2])
  cudaError_t (*prolong_nb[2])(const LevelGeomH &coarse, const VecLayout &lc, const VecLayout &lf,
                               void *fine, const void *coarse_v, void *tmp, cudaStream_t);
  // separate-kernel smoother variants (cross-checks of the fused kernels), per
  // colour: r_I = (b - A x)_I on the interiors of the colour's patches, and
  // x_I <- omega (x_I + A_II^{-1} r_I) with the fast diagonalisation (inv
  // null) or the dense reference-cell inverse inv (interior^2, symmetric)
  cudaError_t (*patch_residual[2][2])(const LevelGeomH &, const VecLayout &, const void *x, const void *b,
                                      void *r, int colour, cudaStream_t);
  cudaError_t (*patch_solve[2][2])(const LevelGeomH &, const VecLayout &, void *x, const void *r,
                                   const void *inv, int colour, double omega, cudaStream_t);
  // x += w a over n entries ([dtype])
  cudaError_t (*scaled_add[2])(void *x, const void *a, double w, int64_t n, cudaStream_t);
};

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda
// link dependency): tiled map of rank 3..5, no swizzle, zero out-of-bounds
// fill; strides_bytes holds the rank-1 strides of dimensions 1.. (dimension
// 0 is contiguous)
cudaError_t encode_tiled(void *map_out, bool f64, void *base, int rank, const uint64_t *dims,
                         const uint64_t *strides_bytes, const uint32_t *box);
inline cudaError_t encode_tiled_3d(void *map_out, bool f64, void *base, const uint64_t dims[3],
                                   const uint64_t strides_bytes[2], const uint32_t box[3])
{
  return encode_tiled(map_out, f64, base, 3, dims, strides_bytes, box);
}

const KernelTable *kernel_table(int degree);

extern const KernelTable kernel_table_k1, kernel_table_k2, kernel_table_k3, kernel_table_k4,
    kernel_table_k5, kernel_table_k6, kernel_table_k7;

// Scale of the stiffness relative to the reference-cell matrices:
// A = h^(dim-2) * sum_d (L (x) M ...) with reference 1D matrices.
inline double stiffness_scale(int dim, double h) { return dim == 2 ? 1.0 : h; }

// number of patches of colour c on a level with n cells per direction
inline void colour_lattice(int dim, int n, int colour, int &nx, int &ny, int &nz, int &count)
{
  const int npd = n - 1;
  auto cnt = [&](int parity) { return npd > parity ? (npd - parity + 1) / 2 : 0; };
  nx = cnt(colour & 1);
  ny = cnt((colour >> 1) & 1);
  nz = dim == 3 ? cnt((colour >> 2) & 1) : 1;
  count = nx * ny * nz;
}

}  // namespace tps
