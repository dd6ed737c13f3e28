// Right-hand-side assembly on the device: b_i = sum over cells and QGauss(k+1)
// points of f(x_q) phi_i(x_q) JxW_q, the loop of
// LaplaceOperator::compute_residual (include/laplace_operator.cuh:118-181, run
// on the host through deal.II's FEValues there) for a general f given at the
// quadrature points.
//
// Layout of f: cells lexicographic (x fastest), then the (k+1)^dim Gauss
// points of the cell lexicographic (x fastest).  On a uniform mesh the
// cell integral is a sum factorisation with the 1D table w_q phi_i(x_q)
// (qwshape) and the factor h^dim.  Cells are added colour by colour (2^dim
// launches over the cells of one parity vector; cells of one colour share no
// DoF), so the sums are deterministic and need no atomics; only interior DoFs
// are written (Dirichlet rows stay zero).  FP64.  One thread per cell: the
// assembly runs once per right-hand side, outside the solve.
#pragma once

#include "tps_common.cuh"

namespace tps {

template <int DIM, int K>
__global__ void __launch_bounds__(128) assemble_rhs_kernel(double *__restrict__ b, const double *__restrict__ fq,
                                                           int n, int64_t sy, int64_t sz, int cx, int cy, int cz,
                                                           int nx, int ny, int count, double hd)
{
  griddep_wait();
  constexpr int NP = K + 1;
  const DegreeTables<K, double> &tb = c_tables<K, double>;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const int jx = t % nx, r = t / nx, jy = r % ny, jz = r / ny;
  const int ex = cx + 2 * jx, ey = cy + 2 * jy, ez = DIM == 3 ? cz + 2 * jz : 0;
  const int64_t cell = DIM == 3 ? (int64_t(ez) * n + ey) * n + ex : int64_t(ey) * n + ex;
  constexpr int NQ = DIM == 3 ? NP * NP * NP : NP * NP;
  const double *f = fq + cell * NQ;
  const int N1 = n * K + 1;
  if constexpr (DIM == 2) {
    // t1[qy][ix] = sum_qx W[qx][ix] f[qy][qx]; out[iy][ix] = sum_qy W[qy][iy] t1[qy][ix]
    double t1[NP][NP];
#pragma unroll
    for (int qy = 0; qy < NP; ++qy)
#pragma unroll
      for (int ix = 0; ix < NP; ++ix) {
        double s = 0.0;
#pragma unroll
        for (int qx = 0; qx < NP; ++qx) s = fmadd(tb.qwshape[qx * NP + ix], f[qy * NP + qx], s);
        t1[qy][ix] = s;
      }
#pragma unroll
    for (int iy = 0; iy < NP; ++iy) {
      const int gy = ey * K + iy;
      if (gy < 1 || gy > N1 - 2) continue;
#pragma unroll
      for (int ix = 0; ix < NP; ++ix) {
        const int gx = ex * K + ix;
        if (gx < 1 || gx > N1 - 2) continue;
        double s = 0.0;
#pragma unroll
        for (int qy = 0; qy < NP; ++qy) s = fmadd(tb.qwshape[qy * NP + iy], t1[qy][ix], s);
        b[gx + gy * sy] += hd * s;
      }
    }
  } else {
    // contract x, then y, then z; one z-plane of quadrature points at a time
    double t2[NP][NP][NP];  // [qz][iy][ix]
#pragma unroll
    for (int qz = 0; qz < NP; ++qz) {
      double t1[NP][NP];  // [qy][ix]
#pragma unroll
      for (int qy = 0; qy < NP; ++qy)
#pragma unroll
        for (int ix = 0; ix < NP; ++ix) {
          double s = 0.0;
#pragma unroll
          for (int qx = 0; qx < NP; ++qx)
            s = fmadd(tb.qwshape[qx * NP + ix], f[(qz * NP + qy) * NP + qx], s);
          t1[qy][ix] = s;
        }
#pragma unroll
      for (int iy = 0; iy < NP; ++iy)
#pragma unroll
        for (int ix = 0; ix < NP; ++ix) {
          double s = 0.0;
#pragma unroll
          for (int qy = 0; qy < NP; ++qy) s = fmadd(tb.qwshape[qy * NP + iy], t1[qy][ix], s);
          t2[qz][iy][ix] = s;
        }
    }
#pragma unroll
    for (int iz = 0; iz < NP; ++iz) {
      const int gz = ez * K + iz;
      if (gz < 1 || gz > N1 - 2) continue;
#pragma unroll
      for (int iy = 0; iy < NP; ++iy) {
        const int gy = ey * K + iy;
        if (gy < 1 || gy > N1 - 2) continue;
#pragma unroll
        for (int ix = 0; ix < NP; ++ix) {
          const int gx = ex * K + ix;
          if (gx < 1 || gx > N1 - 2) continue;
          double s = 0.0;
#pragma unroll
          for (int qz = 0; qz < NP; ++qz) s = fmadd(tb.qwshape[qz * NP + iz], t2[qz][iy][ix], s);
          b[gx + gy * sy + gz * sz] += hd * s;
        }
      }
    }
  }
}

}  // namespace tps
