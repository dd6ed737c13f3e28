// Per-degree launchers.  Included once per translation unit deg<k>.cu with
// TPS_DEGREE defined, so each degree's __constant__ tables live in exactly
// one TU together with every kernel that reads them.
#pragma once

#include <vector>

#include "kernel_table.h"
#include "laplace.cuh"
#include "smoother.cuh"
#include "transfer.cuh"

namespace tps {
namespace {  // one private copy of the launchers per degree TU
namespace deg_impl {

constexpr int K = TPS_DEGREE;

template <typename T>
cudaError_t upload_one(const DegreeData &D)
{
  DegreeTables<K, T> t{};
  constexpr int NP = K + 1, N1 = 2 * K + 1, M = 2 * K - 1;
  for (int i = 0; i < N1 * N1; ++i) {
    t.pmass[i] = static_cast<T>(D.pmass[i]);
    t.plap[i] = static_cast<T>(D.plap[i]);
  }
  for (int i = 0; i < NP * NP; ++i) {
    t.cmass[i] = static_cast<T>(D.cmass[i]);
    t.clap[i] = static_cast<T>(D.clap[i]);
  }
  for (int i = 0; i < M * M; ++i) t.evec[i] = static_cast<T>(D.evec[i]);
  for (int i = 0; i < M; ++i) t.eval[i] = static_cast<T>(D.eval[i]);
  for (int i = 0; i < N1 * NP; ++i) t.prol[i] = static_cast<T>(D.prol[i]);
  return cudaMemcpyToSymbol(c_tables<K, T>, &t, sizeof(t));
}

template <int DIM, typename T>
size_t smoother_smem()
{
  using S = SmootherShape<DIM, K>;
  return sizeof(T) * S::PPB * S::PER_PATCH;
}

template <int DIM, typename T>
size_t laplace_smem()
{
  return sizeof(T) * OpTile<DIM, K>::SMEM_ELEMS;
}

template <typename T>
size_t restrict_smem()
{
  constexpr int C = XYTile<K>::C;
  constexpr int WI = 2 * K * (C + 1) + 1, WO = C * K;
  return sizeof(T) * (WI * WI + WI * WO);
}

template <typename T>
cudaError_t set_attributes()
{
  cudaError_t e;
#define TPS_SET(kern, bytes)                                                             \
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,           \
                           static_cast<int>(bytes));                                    \
  if (e != cudaSuccess) return e;
  TPS_SET((smoother_colour_kernel<2, K, T>), (smoother_smem<2, T>()));
  TPS_SET((smoother_colour_kernel<3, K, T>), (smoother_smem<3, T>()));
  TPS_SET((laplace_kernel<2, K, T, OpMode::Vmult>), (laplace_smem<2, T>()));
  TPS_SET((laplace_kernel<2, K, T, OpMode::Residual>), (laplace_smem<2, T>()));
  TPS_SET((laplace_kernel<3, K, T, OpMode::Vmult>), (laplace_smem<3, T>()));
  TPS_SET((laplace_kernel<3, K, T, OpMode::Residual>), (laplace_smem<3, T>()));
  TPS_SET((restrict_xy_kernel<K, T, XYOut::AddInterior>), (restrict_smem<T>()));
  TPS_SET((restrict_xy_kernel<K, T, XYOut::SetInterior>), (restrict_smem<T>()));
  TPS_SET((restrict_xy_kernel<K, T, XYOut::SetAll>), (restrict_smem<T>()));
#undef TPS_SET
  return cudaSuccess;
}

cudaError_t upload(const DegreeData &D)
{
  cudaError_t e = upload_one<double>(D);
  if (e == cudaSuccess) e = upload_one<float>(D);
  if (e == cudaSuccess) e = set_attributes<double>();
  if (e == cudaSuccess) e = set_attributes<float>();
  return e;
}

template <int DIM, typename T>
cudaError_t laplace(const LevelGeomH &g, void *dst, const void *src, const void *rhs, int mode,
                    cudaStream_t s)
{
  using Tl = OpTile<DIM, K>;
  const dim3 grid(ceil_div(g.n, Tl::CX), ceil_div(g.n, Tl::CY), DIM == 3 ? ceil_div(g.n, Tl::CZ) : 1);
  const T scale = static_cast<T>(stiffness_scale(DIM, g.h));
  const size_t smem = laplace_smem<DIM, T>();
  if (mode == 0)
    laplace_kernel<DIM, K, T, OpMode::Vmult><<<grid, Tl::NT, smem, s>>>(
        static_cast<T *>(dst), static_cast<const T *>(src), nullptr, g.N1, g.n, scale);
  else
    laplace_kernel<DIM, K, T, OpMode::Residual><<<grid, Tl::NT, smem, s>>>(
        static_cast<T *>(dst), static_cast<const T *>(src), static_cast<const T *>(rhs), g.N1,
        g.n, scale);
  return cudaGetLastError();
}

template <int DIM, typename T>
cudaError_t smoother(const LevelGeomH &g, void *x, const void *b, int colour, double omega,
                     cudaStream_t s)
{
  using S = SmootherShape<DIM, K>;
  int nx, ny, nz, count;
  colour_lattice(DIM, g.n, colour, nx, ny, nz, count);
  if (count == 0) return cudaSuccess;
  const double sc = stiffness_scale(DIM, g.h);
  const int cx = colour & 1, cy = (colour >> 1) & 1, cz = (colour >> 2) & 1;
  smoother_colour_kernel<DIM, K, T><<<ceil_div(count, S::PPB), S::NT, smoother_smem<DIM, T>(), s>>>(
      static_cast<T *>(x), static_cast<const T *>(b), g.N1, nx, ny, count, cx, cy, cz,
      static_cast<T>(sc), static_cast<T>(1.0 / sc), static_cast<T>(omega));
  return cudaGetLastError();
}

template <int DIM, typename T>
cudaError_t prolong(const LevelGeomH &gc, void *fine, const void *coarse, void *tmp, cudaStream_t s)
{
  constexpr int C = XYTile<K>::C;
  const int N1c = gc.N1, N1f = 2 * gc.n * K + 1;
  const unsigned gxy = ceil_div(gc.n, C);
  if constexpr (DIM == 2) {
    prolong_xy_kernel<K, T, XYOut::AddInterior><<<dim3(gxy, gxy, 1), XYTile<K>::NT, 0, s>>>(
        static_cast<T *>(fine), static_cast<const T *>(coarse), N1c, N1f, 0, 0, 0, 1);
  } else {
    const int64_t P = static_cast<int64_t>(N1c) * N1c;
    prolong_z_kernel<K, T><<<dim3(ceil_div(P, 256), gc.n), 256, 0, s>>>(
        static_cast<T *>(tmp), static_cast<const T *>(coarse), N1c, N1f, gc.n);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // fine interior planes 1..N1f-2 from tmp planes 1..N1f-2
    prolong_xy_kernel<K, T, XYOut::AddInterior><<<dim3(gxy, gxy, N1f - 2), XYTile<K>::NT, 0, s>>>(
        static_cast<T *>(fine), static_cast<const T *>(tmp), N1c, N1f, P,
        static_cast<int64_t>(N1f) * N1f, 1, 0);
  }
  return cudaGetLastError();
}

template <int DIM, typename T>
cudaError_t restrict_(const LevelGeomH &gc, void *coarse, const void *fine, void *tmp, int add,
                      cudaStream_t s)
{
  constexpr int C = XYTile<K>::C;
  const int N1c = gc.N1, N1f = 2 * gc.n * K + 1;
  const unsigned gxy = ceil_div(gc.n, C);
  const size_t smem = restrict_smem<T>();
  if constexpr (DIM == 2) {
    if (add)
      restrict_xy_kernel<K, T, XYOut::AddInterior><<<dim3(gxy, gxy, 1), XYTile<K>::NT, smem, s>>>(
          static_cast<T *>(coarse), static_cast<const T *>(fine), N1c, N1f, 0, 0, 0, 1);
    else
      restrict_xy_kernel<K, T, XYOut::SetInterior><<<dim3(gxy, gxy, 1), XYTile<K>::NT, smem, s>>>(
          static_cast<T *>(coarse), static_cast<const T *>(fine), N1c, N1f, 0, 0, 0, 1);
  } else {
    const int64_t P = static_cast<int64_t>(N1c) * N1c;
    restrict_xy_kernel<K, T, XYOut::SetAll><<<dim3(gxy, gxy, N1f), XYTile<K>::NT, smem, s>>>(
        static_cast<T *>(tmp), static_cast<const T *>(fine), N1c, N1f,
        static_cast<int64_t>(N1f) * N1f, P, 0, N1f);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (add)
      restrict_z_kernel<K, T, true><<<dim3(ceil_div(P, 256), gc.n), 256, 0, s>>>(
          static_cast<T *>(coarse), static_cast<const T *>(tmp), N1c, N1f);
    else
      restrict_z_kernel<K, T, false><<<dim3(ceil_div(P, 256), gc.n), 256, 0, s>>>(
          static_cast<T *>(coarse), static_cast<const T *>(tmp), N1c, N1f);
  }
  return cudaGetLastError();
}

}  // namespace deg_impl
}  // namespace

#define TPS_CAT_(a, b) a##b
#define TPS_CAT(a, b) TPS_CAT_(a, b)

const KernelTable TPS_CAT(kernel_table_k, TPS_DEGREE) = {
    TPS_DEGREE,
    &deg_impl::upload,
    {{&deg_impl::laplace<2, double>, &deg_impl::laplace<2, float>},
     {&deg_impl::laplace<3, double>, &deg_impl::laplace<3, float>}},
    {{&deg_impl::smoother<2, double>, &deg_impl::smoother<2, float>},
     {&deg_impl::smoother<3, double>, &deg_impl::smoother<3, float>}},
    {{&deg_impl::prolong<2, double>, &deg_impl::prolong<2, float>},
     {&deg_impl::prolong<3, double>, &deg_impl::prolong<3, float>}},
    {{&deg_impl::restrict_<2, double>, &deg_impl::restrict_<2, float>},
     {&deg_impl::restrict_<3, double>, &deg_impl::restrict_<3, float>}},
};

}  // namespace tps
