// Per-degree launchers.  Included once per translation unit deg<k>.cu with
// TPS_DEGREE defined, so each degree's __constant__ tables live in exactly
// one TU together with every kernel that reads them.
#pragma once

#include <vector>

#include "assemble.cuh"
#include "kappa.cuh"
#include "kernel_table.h"
#include "laplace.cuh"
#include "laplace3d_march.cuh"
#include "smoother.cuh"
#include "smoother3d.cuh"
#include "smoother3d_gemm.cuh"
#include "smoother3d_pair.cuh"
#include "smoother3d_pgemm.cuh"
#include "smoother3d_tc.cuh"
#include "smoother3d_warp.cuh"
#include "smoother_variants.cuh"
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
  for (int q = 0; q < NP; ++q)
    for (int i = 0; i < NP; ++i) t.qwshape[q * NP + i] = static_cast<T>(D.qweight[q] * D.qshape[q * NP + i]);
  // folded interior rows of the centro-symmetric patch matrices (FP64, then rounded)
  auto fold = [&](const std::vector<double> &A, T *fe, T *fo) {
    for (int r = 0; r < K; ++r) {
      const int i = r + 1;  // matrix row; r == K-1 is the centre row K
      for (int j = 0; j < K; ++j) {
        fe[r * (K + 1) + j] = static_cast<T>(0.5 * (A[i * N1 + j] + A[i * N1 + N1 - 1 - j]));
        if (r < K - 1) fo[r * K + j] = static_cast<T>(0.5 * (A[i * N1 + j] - A[i * N1 + N1 - 1 - j]));
      }
      fe[r * (K + 1) + K] = static_cast<T>(A[i * N1 + K]);
    }
  };
  fold(D.pmass, t.pmass_fe, t.pmass_fo);
  fold(D.plap, t.plap_fe, t.plap_fo);
  for (int r = 0; r < K - 1; ++r)
    for (int j = 0; j < K; ++j) {
      t.pmass_fp[r * K + j] = Pair<T>::make(t.pmass_fe[r * (K + 1) + j], t.pmass_fo[r * K + j]);
      t.plap_fp[r * K + j] = Pair<T>::make(t.plap_fe[r * (K + 1) + j], t.plap_fo[r * K + j]);
    }
  const int C = K - 1;
  for (int r = 0; r < C; ++r)
    for (int q = 0; q < C; ++q)
      t.evec_p[r * C + q] = Pair<T>::make(t.evec[r * M + q], t.evec[r * M + C + 1 + q]);
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
  TPS_SET((smoother3d_kernel<K, T, true, sm3_variant_ppb<K, T, 0>()>), (Sm3<K, T, sm3_variant_ppb<K, T, 0>()>::BYTES));
  TPS_SET((smoother3d_kernel<K, T, true, sm3_variant_ppb<K, T, 1>()>), (Sm3<K, T, sm3_variant_ppb<K, T, 1>()>::BYTES));
  TPS_SET((smoother3d_kernel<K, T, true, sm3_variant_ppb<K, T, 2>()>), (Sm3<K, T, sm3_variant_ppb<K, T, 2>()>::BYTES));
  TPS_SET((smoother3d_kernel<K, T, false, sm3_variant_ppb<K, T, 0>()>), (Sm3<K, T, sm3_variant_ppb<K, T, 0>()>::BYTES));
  if constexpr (wp3_enabled<K, T>())
    TPS_SET((smoother3d_warp_kernel<K, T, wp3_warps<K, T>()>), (Wp3<K, T, wp3_warps<K, T>()>::BYTES));
  if constexpr (sizeof(T) == 4 && pp3_enabled<K>())
    TPS_SET((smoother3d_pair_kernel<K, pp3_warps<K>()>), (Pp3<K, pp3_warps<K>()>::BYTES));
  TPS_SET((laplace_kernel<2, K, T, OpMode::Vmult>), (laplace_smem<2, T>()));
  TPS_SET((laplace_kernel<2, K, T, OpMode::Residual>), (laplace_smem<2, T>()));
  TPS_SET((laplace3d_march_kernel<K, T, OpMode::Vmult, false>), (sizeof(T) * OpMarch<K, T>::ELEMS));
  TPS_SET((laplace3d_march_kernel<K, T, OpMode::Residual, false>), (sizeof(T) * OpMarch<K, T>::ELEMS));
  // the marching operator is shared-memory heavy: prefer the largest carveout
  e = cudaFuncSetAttribute(laplace3d_march_kernel<K, T, OpMode::Vmult, false>,
                           cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(laplace3d_march_kernel<K, T, OpMode::Residual, false>,
                           cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  if (e != cudaSuccess) return e;
  if constexpr (sizeof(T) == 8) {
    TPS_SET((laplace3d_march_kernel<K, T, OpMode::Vmult, true>), (sizeof(T) * OpMarch<K, T>::ELEMS));
    e = cudaFuncSetAttribute(laplace3d_march_kernel<K, T, OpMode::Vmult, true>,
                             cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e != cudaSuccess) return e;
  }
  TPS_SET((restrict_xy_kernel<K, T, XYOut::AddInterior>), (restrict_smem<T>()));
  TPS_SET((restrict_xy_kernel<K, T, XYOut::SetInterior>), (restrict_smem<T>()));
  TPS_SET((restrict_xy_kernel<K, T, XYOut::SetAll>), (restrict_smem<T>()));
  TPS_SET((kappa_smoother_kernel<2, K, T>), (sizeof(T) * KSm<2, K, T>::ELEMS));
  TPS_SET((patch_residual_kernel<2, K, T>), (sizeof(T) * PVar<2, K>::RES_ELEMS));
  TPS_SET((patch_residual_kernel<3, K, T>), (sizeof(T) * PVar<3, K>::RES_ELEMS));
  TPS_SET((patch_solve_kernel<2, K, T>), (sizeof(T) * PVar<2, K>::SOLVE_ELEMS));
  TPS_SET((patch_solve_kernel<3, K, T>), (sizeof(T) * PVar<3, K>::SOLVE_ELEMS));
  TPS_SET((kappa_smoother_kernel<3, K, T>), (sizeof(T) * KSm<3, K, T>::ELEMS));
#if TPS_DEGREE >= 2
#if TPS_DEGREE >= 5
  // degrees 5..7: the per-patch kernel; 2..4: the patch GEMM below
  if constexpr (sizeof(T) == 4) TPS_SET((smoother3d_tc_kernel<K>), (Tc3<K>::BYTES));
#endif
#if TPS_DEGREE <= 4
  if constexpr (sizeof(T) == 4) TPS_SET((smoother3d_gemm_kernel<K>), (Pg3<K>::BYTES));
#if TPS_DEGREE == 4
  if constexpr (sizeof(T) == 4) {
    TPS_SET((smoother3d_pgemm_kernel<K, 1>), (Pgv<K, 1>::BYTES));
    TPS_SET((smoother3d_pgemm_kernel<K, 3>), (Pgv<K, 3>::BYTES));
  }
#endif
#endif
#endif
#undef TPS_SET
  return cudaSuccess;
}

cudaError_t upload(const DegreeData &D)
{
  cudaError_t e = upload_one<double>(D);
  if (e == cudaSuccess) e = upload_one<float>(D);
#if TPS_DEGREE >= 2 && TPS_DEGREE <= 4
  {
    // built once per process (FP64 dense patch algebra), copied to every device that loads it
    static const std::vector<float> img = patch_gemm_image(D, Pg3<K>::NBE, Pg3<K>::NBO, Pg3<K>::CK);
    if (e == cudaSuccess && img.size() != static_cast<size_t>(Pg3<K>::IMG_FLOATS)) e = cudaErrorInvalidValue;
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_pg3_image<K>, img.data(), sizeof(float) * img.size());
  }
#endif
#if TPS_DEGREE == 4
  {
    // the row-ordered images of the vector-producer kernel: TF32, and TF32 hi/lo
    static const std::vector<float> im1 = patch_gemm_image_ordered(D, Pgv<K, 1>::NBE, Pgv<K, 1>::NBO,
                                                                   Pgv<K, 1>::CK, 1, false);
    static const std::vector<float> im3 = patch_gemm_image_ordered(D, Pgv<K, 3>::NBE, Pgv<K, 3>::NBO,
                                                                   Pgv<K, 3>::CK, 1, true);
    if (e == cudaSuccess && (im1.size() != static_cast<size_t>(Pgv<K, 1>::IMG_FLOATS) ||
                             im3.size() != static_cast<size_t>(Pgv<K, 3>::IMG_FLOATS)))
      e = cudaErrorInvalidValue;
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_pgv_image<K, 1>, im1.data(), sizeof(float) * im1.size());
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_pgv_image<K, 3>, im3.data(), sizeof(float) * im3.size());
  }
#endif
  if (e == cudaSuccess) e = set_attributes<double>();
  if (e == cudaSuccess) e = set_attributes<float>();
  return e;
}

template <int DIM, typename T>
cudaError_t laplace(const LevelGeomH &g, const VecLayout &l, void *dst, const void *src,
                    const void *rhs, int mode, int layers, cudaStream_t s)
{
  const T scale = static_cast<T>(stiffness_scale(DIM, g.h));
  if constexpr (DIM == 3) {
    using Sz = OpMarch<K, T>;
    // at least one CTA per SM of a 148-SM part: 16 layers per CTA on 64^3
    // Q4 (8 on 32^3), 1 on 16^3 and smaller (each CTA recomputes one leading
    // layer; measured, ms per FP64 apply with 4 / 8 / 16 layers: Q4 64^3
    // 0.155 / 0.144 / 0.139, Q7 32^3 0.223 / 0.220 / 0.210; with the earlier
    // streaming kernel, us per apply with 8 layers vs 1: 16^3 24.7 vs 19.5,
    // 8^3 23.0 vs 19.6)
    const int cz = layers > 0 ? layers : opmarch_layers<K, T>(g.n, 148);
    const dim3 grid(ceil_div(g.n, Sz::TX), ceil_div(g.n, Sz::TY), ceil_div(g.n, cz));
    const size_t smem = sizeof(T) * Sz::ELEMS;
    if (mode == 0)
      TPS_LAUNCH((laplace3d_march_kernel<K, T, OpMode::Vmult, false>), grid, Sz::NT, smem, s,
          static_cast<T *>(dst), static_cast<const T *>(src), nullptr, g.N1, g.n, l.sy, l.sz, scale, cz,
          nullptr);
    else
      TPS_LAUNCH((laplace3d_march_kernel<K, T, OpMode::Residual, false>), grid, Sz::NT, smem, s,
          static_cast<T *>(dst), static_cast<const T *>(src), static_cast<const T *>(rhs), g.N1, g.n, l.sy,
          l.sz, scale, cz, nullptr);
  } else {
    using Tl = OpTile<DIM, K>;
    const dim3 grid(ceil_div(g.n, Tl::CX), ceil_div(g.n, Tl::CY), 1);
    const size_t smem = laplace_smem<DIM, T>();
    if (mode == 0)
      TPS_LAUNCH((laplace_kernel<DIM, K, T, OpMode::Vmult>), grid, Tl::NT, smem, s,
          static_cast<T *>(dst), static_cast<const T *>(src), nullptr, g.N1, l.sy, l.sz, scale);
    else
      TPS_LAUNCH((laplace_kernel<DIM, K, T, OpMode::Residual>), grid, Tl::NT, smem, s,
          static_cast<T *>(dst), static_cast<const T *>(src), static_cast<const T *>(rhs), g.N1,
          l.sy, l.sz, scale);
  }
  return cudaGetLastError();
}

// CTAs of `kern` resident per SM (at least 1) and the SM count of the
// current device; the callers keep it in a function-local static, whose
// initialisation is thread-safe
struct Residency {
  int per_sm = 1, n_sm = 1;
};
template <typename... KArgs>
Residency residency(void (*kern)(KArgs...), int threads, size_t smem)
{
  Residency r;
  int dev = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&r.n_sm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || r.n_sm < 1) r.n_sm = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r.per_sm, kern, threads, smem) != cudaSuccess || r.per_sm < 1)
    r.per_sm = 1;
  return r;
}

template <typename T, bool TMA, int PPB>
int sm3_grid(int n_batches)
{
  static const Residency r =
      residency(smoother3d_kernel<K, T, TMA, PPB>, Sm3<K, T, PPB>::NT, Sm3<K, T, PPB>::BYTES);
  const int g = r.per_sm * r.n_sm;
  return n_batches < g ? n_batches : g;
}

// one colour of the 3D sweep with PPB patches per CTA batch (the plain-load
// variant, for vectors without TMA views, always uses the default batch)
template <typename T, int PPB>
void smoother3d_launch(Sm3Args a, const SmootherMaps *maps, void *x, const void *b, T scale, T fd, int *err,
                       cudaStream_t s)
{
  if (maps && maps->valid) {
    using S = Sm3<K, T, PPB>;
    a.n_batches = static_cast<int>(ceil_div(a.n_patches, S::PPB));
    TPS_LAUNCH((smoother3d_kernel<K, T, true, PPB>), sm3_grid<T, true, PPB>(a.n_batches), S::NT, S::BYTES, s,
        *reinterpret_cast<const CUtensorMap *>(maps->x), *reinterpret_cast<const CUtensorMap *>(maps->b),
        static_cast<T *>(x), static_cast<const T *>(b), a, scale, fd, err);
  } else {
    constexpr int P0 = sm3_variant_ppb<K, T, 0>();
    using S = Sm3<K, T, P0>;
    a.n_batches = static_cast<int>(ceil_div(a.n_patches, S::PPB));
    CUtensorMap none{};
    TPS_LAUNCH((smoother3d_kernel<K, T, false, P0>), a.n_batches, S::NT, S::BYTES, s,
        none, none, static_cast<T *>(x), static_cast<const T *>(b), a, scale, fd, err);
  }
}

// one colour with one patch per team of warps (TMA views required): a
// persistent grid of the CTAs resident per SM x SMs, capped by the patch count
template <typename T>
void smoother3d_warp_launch(const Sm3Args &a, const SmootherMaps *maps, void *x, T scale, T fd, int *err,
                            cudaStream_t s)
{
  if constexpr (wp3_enabled<K, T>()) {
    constexpr int WA = wp3_warps<K, T>();
    using S = Wp3<K, T, WA>;
    static const Residency r = residency(smoother3d_warp_kernel<K, T, WA>, S::NT, S::BYTES);
    const int need = a.n_patches;  // one patch at a time per CTA
    const int grid = need < r.per_sm * r.n_sm ? need : r.per_sm * r.n_sm;
    TPS_LAUNCH((smoother3d_warp_kernel<K, T, WA>), grid, S::NT, S::BYTES, s,
        *reinterpret_cast<const CUtensorMap *>(maps->x), *reinterpret_cast<const CUtensorMap *>(maps->b),
        static_cast<T *>(x), a, scale, fd, err);
  }
}

// one colour with two patches per warp in packed FP32 (TMA views required):
// a persistent grid of the CTAs resident per SM x SMs, capped by the pair count
// (a grid sized so that every CTA takes the same number of pairs, at fewer
// CTAs per SM, measured slower: 0.471 against 0.452 ms per Q4 64^3 sweep)
void smoother3d_pair_launch(const Sm3Args &a, const SmootherMaps *maps, void *x, float scale, float fd, int *err,
                            cudaStream_t s)
{
  if constexpr (pp3_enabled<K>()) {
    constexpr int WA = pp3_warps<K>();
    using S = Pp3<K, WA>;
    static_assert(S::BYTES + 1024 <= 233472, "pair smoother: one CTA must fit an SM");
    static const Residency r = residency(smoother3d_pair_kernel<K, WA>, S::NT, S::BYTES);
    const int need = static_cast<int>(ceil_div(a.n_patches, 2));  // one pair at a time per CTA
    const int grid = need < r.per_sm * r.n_sm ? need : r.per_sm * r.n_sm;
    TPS_LAUNCH((smoother3d_pair_kernel<K, WA>), grid, S::NT, S::BYTES, s,
        *reinterpret_cast<const CUtensorMap *>(maps->x), *reinterpret_cast<const CUtensorMap *>(maps->b),
        static_cast<float *>(x), a, scale, fd, err);
  }
}

// patches per batch of a 3D variant (0 in 2D: one fixed kernel shape; -1:
// the one-warp-per-patch kernel, variant 3, -2: two patches per warp in
// packed FP32, variant 4, where they are compiled)
int smoother_ppb(int dim, int dtype, int variant)
{
  if (dim != 3) return 0;
  auto pick = [&](auto tag) -> int {
    using T = decltype(tag);
    if (variant == 4) return (sizeof(T) == 4 && pp3_enabled<K>()) ? -2 : sm3_variant_ppb<K, T, 0>();
    if (variant == 3) return wp3_enabled<K, T>() ? -1 : sm3_variant_ppb<K, T, 0>();
    return variant == 1 ? sm3_variant_ppb<K, T, 1>() : variant == 2 ? sm3_variant_ppb<K, T, 2>()
                                                                        : sm3_variant_ppb<K, T, 0>();
  };
  return dtype == 0 ? pick(double{}) : pick(float{});
}

template <int DIM, typename T>
cudaError_t smoother(const LevelGeomH &g, const VecLayout &l, void *x, const void *b, int colour,
                     double omega, int zero_x, int variant, const SmootherMaps *maps, int *err, cudaStream_t s)
{
  int nx, ny, nz, count;
  colour_lattice(DIM, g.n, colour, nx, ny, nz, count);
  if (count == 0) return cudaSuccess;
  const double sc = stiffness_scale(DIM, g.h);
  const int cx = colour & 1, cy = (colour >> 1) & 1, cz = (colour >> 2) & 1;
  if constexpr (DIM == 2) {
    using S = SmootherShape<DIM, K>;
    (void)zero_x;  // the 2D kernel always reads x (x == 0 gives the same sweep)
    (void)maps;
    (void)err;
    TPS_LAUNCH((smoother_colour_kernel<DIM, K, T>), ceil_div(count, S::PPB), S::NT, smoother_smem<DIM, T>(), s,
        static_cast<T *>(x), static_cast<const T *>(b), l.sy, l.sz, nx, ny, count, cx, cy, cz,
        static_cast<T>(sc), static_cast<T>(1.0 / sc), static_cast<T>(omega));
  } else {
    Sm3Args a;
    a.nx_c = nx;
    a.ny_c = ny;
    a.n_patches = count;
    a.cx = cx;
    a.cy = cy;
    a.cz = cz;
    a.zero_x = zero_x;
    a.sy = l.sy;
    a.sz = l.sz;
    magic_div(static_cast<uint32_t>(nx), a.mx, a.sx);
    magic_div(static_cast<uint32_t>(nx) * static_cast<uint32_t>(ny), a.mxy, a.sxy);
    const T scale = static_cast<T>(sc), fd = static_cast<T>(omega / sc);
    bool pair = false;
    if constexpr (sizeof(T) == 4) pair = variant == 4 && pp3_enabled<K>() && maps && maps->valid;
    if (pair)
      smoother3d_pair_launch(a, maps, x, static_cast<float>(scale), static_cast<float>(fd), err, s);
    else if (variant == 3 && wp3_enabled<K, T>() && maps && maps->valid)
      smoother3d_warp_launch<T>(a, maps, x, scale, fd, err, s);
    else if (variant == 1)
      smoother3d_launch<T, sm3_variant_ppb<K, T, 1>()>(a, maps, x, b, scale, fd, err, s);
    else if (variant == 2)
      smoother3d_launch<T, sm3_variant_ppb<K, T, 2>()>(a, maps, x, b, scale, fd, err, s);
    else
      smoother3d_launch<T, sm3_variant_ppb<K, T, 0>()>(a, maps, x, b, scale, fd, err, s);
  }
  return cudaGetLastError();
}

#if TPS_DEGREE >= 2
#if TPS_DEGREE >= 5
// persistent grid of the per-patch tensor-core smoother: CTAs resident per SM
// x SMs, capped so that every CTA's TMEM allocation fits at once
int tc_grid(int n_units)
{
  {
    using C = Tc3<K>;
    static const Residency r = [] {
      Residency q = residency(smoother3d_tc_kernel<K>, C::NT, C::BYTES);
      if (q.per_sm * C::TMEM_COLS > 512) q.per_sm = 512 / C::TMEM_COLS;  // every CTA's TMEM fits at once
      return q;
    }();
    const int g = r.per_sm * r.n_sm;
    return n_units < g ? n_units : g;
  }
}
#endif

cudaError_t smoother_tc(const LevelGeomH &g, const VecLayout &l, void *x, const void *b, int colour,
                        double omega, int zero_x, const SmootherMaps *maps, int passes, int *err, cudaStream_t s)
{
#if TPS_DEGREE != 4
  if (passes != 1) return cudaErrorNotSupported;
#endif
#if TPS_DEGREE <= 4
  {
    // degrees 2..4: the patch step as one GEMM over the colour's patches
    int nx, ny, nz, count;
    colour_lattice(3, g.n, colour, nx, ny, nz, count);
    if (count == 0) return cudaSuccess;
    const double sc = stiffness_scale(3, g.h);
    Sm3Args a;
    a.nx_c = nx;
    a.ny_c = ny;
    a.n_patches = count;
    a.cx = colour & 1;
    a.cy = (colour >> 1) & 1;
    a.cz = (colour >> 2) & 1;
    a.n_batches = count;
    a.zero_x = zero_x;
    a.sy = l.sy;
    a.sz = l.sz;
    magic_div(static_cast<uint32_t>(nx), a.mx, a.sx);
    magic_div(static_cast<uint32_t>(nx) * static_cast<uint32_t>(ny), a.mxy, a.sxy);
    // one CTA per SM (its shared memory and TMEM allow no second)
    static const int n_sm = [] {
      int dev = 0, n = 0;
      cudaGetDevice(&dev);
      return cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && n > 0 ? n : 1;
    }();
    const int tiles = static_cast<int>(ceil_div(count, 128));
    const int grid = tiles < n_sm ? tiles : n_sm;
#if TPS_DEGREE == 4
    // the vector-producer kernel reads box rows as 16-byte vectors: vectors
    // and pitches aligned to 4 entries (always true for the V-cycle's padded
    // work vectors)
    const bool vec_ok = (reinterpret_cast<uintptr_t>(x) % 16 == 0) && (reinterpret_cast<uintptr_t>(b) % 16 == 0) &&
                        l.sy % 4 == 0 && l.sz % 4 == 0;
    if (passes == 3 && !vec_ok) return cudaErrorNotSupported;
    // one TF32 pass: the gather kernel below measured faster (0.511 vs 0.763 ms
    // per Q4 64^3 sweep); the vector-producer kernel serves the three-pass split
    if (vec_ok && passes == 3) {
      if (passes == 3)
        TPS_LAUNCH((smoother3d_pgemm_kernel<K, 3>), grid, (Pgv<K, 3>::NT), (Pgv<K, 3>::BYTES), s,
            static_cast<float *>(x), static_cast<const float *>(b), a, static_cast<float>(sc),
            static_cast<float>(omega / sc), err);
      else
        TPS_LAUNCH((smoother3d_pgemm_kernel<K, 1>), grid, (Pgv<K, 1>::NT), (Pgv<K, 1>::BYTES), s,
            static_cast<float *>(x), static_cast<const float *>(b), a, static_cast<float>(sc),
            static_cast<float>(omega / sc), err);
      return cudaGetLastError();
    }
#endif
    TPS_LAUNCH((smoother3d_gemm_kernel<K>), grid, Pg3<K>::NT, Pg3<K>::BYTES, s,
        static_cast<float *>(x), static_cast<const float *>(b), a, static_cast<float>(sc),
        static_cast<float>(omega / sc), err);
    (void)maps;
    return cudaGetLastError();
  }
#else
  {
    using C = Tc3<K>;
    if (!maps || !maps->tc_valid) return cudaErrorInvalidValue;
    int nx, ny, nz, count;
    colour_lattice(3, g.n, colour, nx, ny, nz, count);
    if (count == 0) return cudaSuccess;
    const double sc = stiffness_scale(3, g.h);
    Sm3Args a;
    a.nx_c = nx;
    a.ny_c = ny;
    a.n_patches = count;
    a.cx = colour & 1;
    a.cy = (colour >> 1) & 1;
    a.cz = (colour >> 2) & 1;
    a.n_batches = count;
    a.zero_x = zero_x;
    a.sy = l.sy;
    a.sz = l.sz;
    magic_div(static_cast<uint32_t>(nx), a.mx, a.sx);
    magic_div(static_cast<uint32_t>(nx) * static_cast<uint32_t>(ny), a.mxy, a.sxy);
    TPS_LAUNCH((smoother3d_tc_kernel<K>), tc_grid(static_cast<int>(ceil_div(count, C::U))), C::NT, C::BYTES, s,
        *reinterpret_cast<const CUtensorMap *>(maps->tx), *reinterpret_cast<const CUtensorMap *>(maps->tb),
        static_cast<float *>(x), a, static_cast<float>(sc), static_cast<float>(omega / sc), err);
    return cudaGetLastError();
  }
#endif
}

cudaError_t encode_tc_maps(const VecLayout &l, void *x, const void *b, SmootherMaps *out)
{
  out->tc_valid = 0;
  {
    using C = Tc3<K>;
    if ((l.sy * 4) % 16 || (l.sz * 4) % 16 || reinterpret_cast<uintptr_t>(x) % 16 ||
        reinterpret_cast<uintptr_t>(b) % 16)
      return cudaSuccess;
    const uint64_t N = static_cast<uint64_t>(l.N1), NC = (N + 3) / 4;
    const uint64_t sy = static_cast<uint64_t>(l.sy) * 4, sz = static_cast<uint64_t>(l.sz) * 4;
    // x: (x%4, y, x/4, z), 8 rows of y per load -> [z][x/4][y%8][x%4] (K-major, K = x)
    const uint64_t dx[4] = {4, N, NC, N}, stx[3] = {sy, 16, sz};
    const uint32_t bx[4] = {4, 8, static_cast<uint32_t>(C::XC), static_cast<uint32_t>(C::N1)};
    // b: plain [z][y][x] box of the patch interior (x from the aligned box start)
    const uint64_t db[3] = {N, N, N}, stb[2] = {sy, sz};
    const uint32_t bb[3] = {static_cast<uint32_t>(C::XW), static_cast<uint32_t>(C::M), static_cast<uint32_t>(C::M)};
    cudaError_t e = encode_tiled(out->tx, false, x, 4, dx, stx, bx);
    if (e == cudaSuccess) e = encode_tiled(out->tb, false, const_cast<void *>(b), 3, db, stb, bb);
    if (e == cudaSuccess) out->tc_valid = 1;
    return e;
  }
}

#else
cudaError_t encode_tc_maps(const VecLayout &, void *, const void *, SmootherMaps *out)
{
  out->tc_valid = 0;
  return cudaSuccess;
}
#endif

template <typename T>
cudaError_t encode_maps(const VecLayout &l, void *x, const void *b, SmootherMaps *out)
{
  using S = Sm3<K, T>;
  out->valid = 0;
  const uint64_t es = sizeof(T);
  if ((l.sy * es) % 16 || (l.sz * es) % 16 || reinterpret_cast<uintptr_t>(x) % 16 ||
      reinterpret_cast<uintptr_t>(b) % 16)
    return cudaSuccess;  // pitch not TMA-compatible: the plain-load variant is used
  const uint64_t dims[3] = {static_cast<uint64_t>(l.N1), static_cast<uint64_t>(l.N1),
                            static_cast<uint64_t>(l.N1)};
  const uint64_t str[2] = {static_cast<uint64_t>(l.sy) * es, static_cast<uint64_t>(l.sz) * es};
  const uint32_t bx[3] = {S::W, S::N1, S::N1}, bb[3] = {S::W, S::M, S::M};
  cudaError_t e = encode_tiled_3d(out->x, sizeof(T) == 8, x, dims, str, bx);
  if (e == cudaSuccess) e = encode_tiled_3d(out->b, sizeof(T) == 8, const_cast<void *>(b), dims, str, bb);
  if (e == cudaSuccess) out->valid = 1;
  return e;
}

template <int DIM, typename T, bool MASK>
cudaError_t prolong_impl(const LevelGeomH &gc, const VecLayout &lc, const VecLayout &lf, void *fine,
                         const void *coarse, void *tmp, cudaStream_t s)
{
  constexpr int C = ProlTile<K, T>::C;
  const int N1c = gc.N1, N1f = 2 * gc.n * K + 1;
  const unsigned gxy = ceil_div(gc.n, C);
  if constexpr (DIM == 2) {
    TPS_LAUNCH((prolong_xy_kernel<K, T, XYOut::AddInterior>), dim3(gxy, gxy, 1), XYTile<K>::NT, 0, s,
        static_cast<T *>(fine), static_cast<const T *>(coarse), N1c, N1f, lc.sy, 0, lf.sy, 0, 0, MASK ? 1 : 0);
  } else {
    const int64_t P = static_cast<int64_t>(N1c) * N1c;
    TPS_LAUNCH((prolong_z_kernel<K, T, MASK>), dim3(ceil_div(P, 256), gc.n), 256, 0, s,
        static_cast<T *>(tmp), static_cast<const T *>(coarse), N1c, N1f, gc.n, lc.sy, lc.sz);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // fine interior planes 1..N1f-2 from tmp planes 1..N1f-2
    TPS_LAUNCH((prolong_xy_kernel<K, T, XYOut::AddInterior>), dim3(gxy, gxy, N1f - 2), XYTile<K>::NT, 0, s,
        static_cast<T *>(fine), static_cast<const T *>(tmp), N1c, N1f, N1c, P, lf.sy, lf.sz, 1, MASK ? 1 : 0);
  }
  return cudaGetLastError();
}

template <int DIM, typename T>
cudaError_t prolong(const LevelGeomH &gc, const VecLayout &lc, const VecLayout &lf, void *fine,
                    const void *coarse, void *tmp, cudaStream_t s)
{
  return prolong_impl<DIM, T, true>(gc, lc, lf, fine, coarse, tmp, s);
}

// FP64 prolongation that reads the coarse boundary values (the FMG
// prolongation of the solution); fine interior DoFs += P coarse
template <int DIM>
cudaError_t prolong_nb(const LevelGeomH &gc, const VecLayout &lc, const VecLayout &lf, void *fine,
                       const void *coarse, void *tmp, cudaStream_t s)
{
  return prolong_impl<DIM, double, false>(gc, lc, lf, fine, coarse, tmp, s);
}

template <int DIM, typename T>
cudaError_t restrict_(const LevelGeomH &gc, const VecLayout &lc, const VecLayout &lf, void *coarse,
                      const void *fine, void *tmp, int add, cudaStream_t s)
{
  constexpr int C = XYTile<K>::C;
  const int N1c = gc.N1, N1f = 2 * gc.n * K + 1;
  const unsigned gxy = ceil_div(gc.n, C);
  const size_t smem = restrict_smem<T>();
  if constexpr (DIM == 2) {
    if (add)
      TPS_LAUNCH((restrict_xy_kernel<K, T, XYOut::AddInterior>), dim3(gxy, gxy, 1), XYTile<K>::NT, smem, s,
          static_cast<T *>(coarse), static_cast<const T *>(fine), N1c, N1f, lf.sy, 0, lc.sy, 0, 0, 1);
    else
      TPS_LAUNCH((restrict_xy_kernel<K, T, XYOut::SetInterior>), dim3(gxy, gxy, 1), XYTile<K>::NT, smem, s,
          static_cast<T *>(coarse), static_cast<const T *>(fine), N1c, N1f, lf.sy, 0, lc.sy, 0, 0, 1);
  } else {
    const int64_t P = static_cast<int64_t>(N1c) * N1c;
    TPS_LAUNCH((restrict_xy_kernel<K, T, XYOut::SetAll>), dim3(gxy, gxy, N1f), XYTile<K>::NT, smem, s,
        static_cast<T *>(tmp), static_cast<const T *>(fine), N1c, N1f, lf.sy, lf.sz, N1c, P, 0, N1f);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (add)
      TPS_LAUNCH((restrict_z_kernel<K, T, true>), dim3(ceil_div(P, 256), gc.n), 256, 0, s,
          static_cast<T *>(coarse), static_cast<const T *>(tmp), N1c, N1f, lc.sy, lc.sz);
    else
      TPS_LAUNCH((restrict_z_kernel<K, T, false>), dim3(ceil_div(P, 256), gc.n), 256, 0, s,
          static_cast<T *>(coarse), static_cast<const T *>(tmp), N1c, N1f, lc.sy, lc.sz);
  }
  return cudaGetLastError();
}

// cells of colour c: parities of (cx, cy, cz)
inline void cell_lattice(int dim, int n, int colour, int &nx, int &ny, int &nz)
{
  auto cnt = [&](int parity) { return n > parity ? (n - parity + 1) / 2 : 0; };
  nx = cnt(colour & 1);
  ny = cnt((colour >> 1) & 1);
  nz = dim == 3 ? cnt((colour >> 2) & 1) : 1;
}

template <int DIM, typename T, bool MASS>
cudaError_t cell_sweep(const LevelGeomH &g, const VecLayout &l, T *dst, const T *src, const T *kappa,
                       double s, cudaStream_t st)
{
  for (int c = 0; c < (1 << DIM); ++c) {
    int nx, ny, nz;
    cell_lattice(DIM, g.n, c, nx, ny, nz);
    const int count = nx * ny * nz;
    if (count == 0) continue;
    TPS_LAUNCH((cell_apply_kernel<DIM, K, T, MASS>), count, KappaCfg<DIM, K>::NT, 0, st,
        dst, src, kappa, g.n, c, nx, ny, l.sy, l.sz, static_cast<T>(s));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <int DIM, typename T>
cudaError_t kappa_laplace(const LevelGeomH &g, const VecLayout &l, void *dst, const void *src,
                          const void *rhs, const void *kappa, int mode, cudaStream_t st)
{
  const int64_t n = DIM == 3 ? l.sz * g.N1 : l.sy * g.N1;
  cudaError_t e = cudaMemsetAsync(dst, 0, sizeof(T) * n, st);
  if (e != cudaSuccess) return e;
  e = cell_sweep<DIM, T, false>(g, l, static_cast<T *>(dst), static_cast<const T *>(src),
                                static_cast<const T *>(kappa), stiffness_scale(DIM, g.h), st);
  if (e != cudaSuccess) return e;
  // Dirichlet rows end at 0 like the unit-coefficient kernel's untouched rows
  // of zero-initialised work vectors; tps_laplace_vmult then copies src there
  TPS_LAUNCH((finish_residual_kernel<DIM, T>), 1184, 256, 0, st,
      static_cast<T *>(dst), mode == 1 ? static_cast<const T *>(rhs) : nullptr, g.N1, l.sy, l.sz);
  return cudaGetLastError();
}

template <int DIM, typename T>
cudaError_t kappa_smoother(const LevelGeomH &g, const VecLayout &l, void *x, const void *b,
                           const void *kappa, int colour, double omega, cudaStream_t st)
{
  int nx, ny, nz, count;
  colour_lattice(DIM, g.n, colour, nx, ny, nz, count);
  if (count == 0) return cudaSuccess;
  const double sc = stiffness_scale(DIM, g.h);
  TPS_LAUNCH((kappa_smoother_kernel<DIM, K, T>), count, KSm<DIM, K, T>::NT, sizeof(T) * KSm<DIM, K, T>::ELEMS, st,
      static_cast<T *>(x), static_cast<const T *>(b), static_cast<const T *>(kappa), g.n, colour,
      nx, ny, l.sy, l.sz, static_cast<T>(sc), static_cast<T>(1.0 / sc), static_cast<T>(omega));
  return cudaGetLastError();
}

template <int DIM>
cudaError_t mass(const LevelGeomH &g, const VecLayout &l, double *dst, const double *src, cudaStream_t st)
{
  const int64_t n = DIM == 3 ? l.sz * g.N1 : l.sy * g.N1;
  cudaError_t e = cudaMemsetAsync(dst, 0, sizeof(double) * n, st);
  if (e != cudaSuccess) return e;
  double hd = 1.0;
  for (int d = 0; d < DIM; ++d) hd *= g.h;
  return cell_sweep<DIM, double, true>(g, l, dst, src, nullptr, hd, st);
}

// b = sum over cells and Gauss points of f phi_i JxW (interior rows; b zeroed first)
// 3D FP64 q = A p with the CG's p.q partial sums fused (one per CTA into
// partial, at most `capacity`; *ctas receives their count)
cudaError_t laplace3d_dot(const LevelGeomH &g, const VecLayout &l, void *dst, const void *src, double *partial,
                          int capacity, int layers, int *ctas, cudaStream_t s)
{
  using Sz = OpMarch<K, double>;
  const int cz = layers > 0 ? layers : opmarch_layers<K, double>(g.n, 148);
  const dim3 grid(ceil_div(g.n, Sz::TX), ceil_div(g.n, Sz::TY), ceil_div(g.n, cz));
  const int64_t count = int64_t(grid.x) * grid.y * grid.z;
  if (count > capacity) return cudaErrorInvalidValue;
  *ctas = static_cast<int>(count);
  TPS_LAUNCH((laplace3d_march_kernel<K, double, OpMode::Vmult, true>), grid, Sz::NT, sizeof(double) * Sz::ELEMS,
      s, static_cast<double *>(dst), static_cast<const double *>(src), nullptr, g.N1, g.n, l.sy, l.sz,
      stiffness_scale(3, g.h), cz, partial);
  return cudaGetLastError();
}

// the most CTAs laplace3d_dot launches on a level of n cells (one layer per CTA)
int laplace3d_ctas(int n)
{
  using Sz = OpMarch<K, double>;
  return ceil_div(n, Sz::TX) * ceil_div(n, Sz::TY) * n;
}

template <int DIM>
cudaError_t assemble_rhs(const LevelGeomH &g, const VecLayout &l, double *b, const double *fq, cudaStream_t st)
{
  const int64_t n = DIM == 3 ? l.sz * g.N1 : l.sy * g.N1;
  cudaError_t e = cudaMemsetAsync(b, 0, sizeof(double) * n, st);
  if (e != cudaSuccess) return e;
  double hd = 1.0;
  for (int d = 0; d < DIM; ++d) hd *= g.h;
  for (int c = 0; c < (1 << DIM); ++c) {
    const int cx = c & 1, cy = (c >> 1) & 1, cz = (c >> 2) & 1;
    const int nx = (g.n - cx + 1) / 2, ny = (g.n - cy + 1) / 2, nz = DIM == 3 ? (g.n - cz + 1) / 2 : 1;
    const int count = nx * ny * nz;
    if (count == 0) continue;
    TPS_LAUNCH((assemble_rhs_kernel<DIM, K>), static_cast<unsigned>(ceil_div(count, 128)), 128, 0, st, b, fq, g.n,
        l.sy, l.sz, cx, cy, cz, nx, ny, count, hd);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <int DIM>
cudaError_t cell_energy(const LevelGeomH &g, const VecLayout &l, double *e, const double *u,
                        const double *lam, cudaStream_t st)
{
  const int64_t ncell = DIM == 3 ? int64_t(g.n) * g.n * g.n : int64_t(g.n) * g.n;
  TPS_LAUNCH((cell_energy_kernel<DIM, K>), static_cast<unsigned>(ncell), KappaCfg<DIM, K>::NT, 0, st,
      e, u, lam, g.n, l.sy, l.sz, stiffness_scale(DIM, g.h));
  return cudaGetLastError();
}

// patches of colour `colour` of a level with layout l
template <int DIM>
PatchColour patch_colour(const LevelGeomH &g, const VecLayout &l, int colour)
{
  PatchColour c;
  int nz = 1;
  colour_lattice(DIM, g.n, colour, c.nx, c.ny, nz, c.count);
  c.cx = colour & 1;
  c.cy = (colour >> 1) & 1;
  c.cz = (colour >> 2) & 1;
  c.sy = l.sy;
  c.sz = l.sz;
  return c;
}

template <int DIM, typename T>
cudaError_t patch_residual(const LevelGeomH &g, const VecLayout &l, const void *x, const void *b, void *r,
                           int colour, cudaStream_t s)
{
  const PatchColour c = patch_colour<DIM>(g, l, colour);
  if (c.count == 0) return cudaSuccess;
  using S = PVar<DIM, K>;
  TPS_LAUNCH((patch_residual_kernel<DIM, K, T>), c.count, S::NT, sizeof(T) * S::RES_ELEMS, s,
      static_cast<const T *>(x), static_cast<const T *>(b), static_cast<T *>(r), c,
      static_cast<T>(stiffness_scale(DIM, g.h)));
  return cudaGetLastError();
}

template <int DIM, typename T>
cudaError_t patch_solve(const LevelGeomH &g, const VecLayout &l, void *x, const void *r, const void *inv,
                        int colour, double omega, cudaStream_t s)
{
  const PatchColour c = patch_colour<DIM>(g, l, colour);
  if (c.count == 0) return cudaSuccess;
  using S = PVar<DIM, K>;
  TPS_LAUNCH((patch_solve_kernel<DIM, K, T>), c.count, S::NT, sizeof(T) * S::SOLVE_ELEMS, s,
      static_cast<T *>(x), static_cast<const T *>(r), static_cast<const T *>(inv), c, static_cast<T>(omega),
      static_cast<T>(1.0 / stiffness_scale(DIM, g.h)));
  return cudaGetLastError();
}

template <typename T>
cudaError_t scaled_add(void *x, const void *a, double w, int64_t n, cudaStream_t s)
{
  const int64_t blocks = (n + 255) / 256;
  TPS_LAUNCH((scaled_add_kernel<T>), static_cast<unsigned>(blocks < 4 * 148 ? blocks : 4 * 148), 256, 0, s,
             static_cast<T *>(x), static_cast<const T *>(a), static_cast<T>(w), n);
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
    {&deg_impl::encode_maps<double>, &deg_impl::encode_maps<float>},
    {{&deg_impl::prolong<2, double>, &deg_impl::prolong<2, float>},
     {&deg_impl::prolong<3, double>, &deg_impl::prolong<3, float>}},
    {{&deg_impl::restrict_<2, double>, &deg_impl::restrict_<2, float>},
     {&deg_impl::restrict_<3, double>, &deg_impl::restrict_<3, float>}},
    {{&deg_impl::kappa_laplace<2, double>, &deg_impl::kappa_laplace<2, float>},
     {&deg_impl::kappa_laplace<3, double>, &deg_impl::kappa_laplace<3, float>}},
    {{&deg_impl::kappa_smoother<2, double>, &deg_impl::kappa_smoother<2, float>},
     {&deg_impl::kappa_smoother<3, double>, &deg_impl::kappa_smoother<3, float>}},
    {&deg_impl::mass<2>, &deg_impl::mass<3>},
    {&deg_impl::cell_energy<2>, &deg_impl::cell_energy<3>},
    {&deg_impl::assemble_rhs<2>, &deg_impl::assemble_rhs<3>},
    &deg_impl::laplace3d_dot,
    &deg_impl::laplace3d_ctas,
#if TPS_DEGREE >= 2
    &deg_impl::smoother_tc,
#else
    nullptr,
#endif
    &deg_impl::encode_tc_maps,
    &deg_impl::smoother_ppb,
    {&deg_impl::prolong_nb<2>, &deg_impl::prolong_nb<3>},
    {{&deg_impl::patch_residual<2, double>, &deg_impl::patch_residual<2, float>},
     {&deg_impl::patch_residual<3, double>, &deg_impl::patch_residual<3, float>}},
    {{&deg_impl::patch_solve<2, double>, &deg_impl::patch_solve<2, float>},
     {&deg_impl::patch_solve<3, double>, &deg_impl::patch_solve<3, float>}},
    {&deg_impl::scaled_add<double>, &deg_impl::scaled_add<float>},
};

}  // namespace tps
