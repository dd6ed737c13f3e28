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

struct KernelTable {
  int degree;
  // copy the 1D tables of this degree into constant memory of the current device
  cudaError_t (*upload)(const DegreeData &);
  // dst = A src on interior rows (mode 0) or dst = rhs - A src (mode 1);
  // boundary rows of dst are not written
  cudaError_t (*laplace[2][2])(const LevelGeomH &, void *dst, const void *src, const void *rhs,
                               int mode, cudaStream_t);
  // one colour of the patch sweep
  cudaError_t (*smoother[2][2])(const LevelGeomH &, void *x, const void *b, int colour,
                                double omega, cudaStream_t);
  // fine += P coarse (interior fine DoFs); geometry of the COARSE level
  cudaError_t (*prolong[2][2])(const LevelGeomH &coarse, void *fine, const void *coarse_v,
                               void *tmp, cudaStream_t);
  // coarse (+)= R fine on interior coarse DoFs; geometry of the COARSE level
  cudaError_t (*restrict_[2][2])(const LevelGeomH &coarse, void *coarse_v, const void *fine,
                                 void *tmp, int add, cudaStream_t);
};

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
