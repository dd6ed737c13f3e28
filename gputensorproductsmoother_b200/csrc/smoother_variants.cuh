// Separate-kernel patch smoother variants: cross-checks of the fused kernels.
//
// Reference: LevelVertexPatch::patch_loop_seperate / patch_loop_global
// (include/patch_base.template.cuh:545-707) with loop_kernel_seperate and
// loop_kernel_seperate_inv (include/loop_kernel.cuh:54-578), the Exact local
// solver (include/loop_kernel.cuh:241-327), dispatched by
// PatchSmootherImpl::step_impl (include/patch_smoother.cuh:185-260).  For
// every colour:
//   1. r_I = (b - A x)_I on the interiors of the colour's patches, from each
//      patch box (SEPERATE, Exact: patch_residual_kernel) or from the global
//      operator (GLOBAL: the level operator in residual mode);
//   2. x_I <- omega (x_I + A_II^{-1} r_I) per patch (patch_solve_kernel), with
//      the fast diagonalisation S Lambda^{-1} S^T (SEPERATE, GLOBAL) or with
//      the dense inverse of the assembled interior patch matrix (Exact).
// One CTA per patch with plain loads and dense 1D patch matrices staged in
// shared memory: an implementation independent of the fused kernels
// (folded constant-bank contractions, TMA staging, zero-interior algebra), so
// that agreement of the two checks both.
#pragma once

#include "tps_common.cuh"

namespace tps {

// patches of one colour: lattice extents, parities and the vector layout
struct PatchColour {
  int nx, ny, count;
  int cx, cy, cz;
  int64_t sy, sz;
};

template <int DIM, int K>
struct PVar {
  static constexpr int N1 = 2 * K + 1, M = 2 * K - 1;
  static constexpr int BOX = DIM == 3 ? N1 * N1 * N1 : N1 * N1;
  static constexpr int INT = DIM == 3 ? M * M * M : M * M;
  static constexpr int NT = 128;
  // residual: Pm | Pl | X[BOX] | Z1 | Z2 | V1 | V2 (3D)
  static constexpr int ZS = DIM == 3 ? M * N1 * N1 : M * N1;
  static constexpr int VS = DIM == 3 ? M * M * N1 : 0;
  static constexpr int RES_ELEMS = 2 * N1 * N1 + BOX + 2 * ZS + 2 * VS;
  // solve: Ev | lambda | Q0 | Q1
  static constexpr int SOLVE_ELEMS = M * M + M + 2 * INT;
};

// global index of the first (corner) DoF of patch j of the colour
template <int DIM, int K>
__device__ __forceinline__ int64_t pv_origin(const PatchColour &c, int j)
{
  const int jx = j % c.nx;
  const int jy = DIM == 3 ? (j / c.nx) % c.ny : j / c.nx;
  const int jz = DIM == 3 ? j / (c.nx * c.ny) : 0;
  return static_cast<int64_t>(c.cx + 2 * jx) * K + static_cast<int64_t>(c.cy + 2 * jy) * K * c.sy +
         (DIM == 3 ? static_cast<int64_t>(c.cz + 2 * jz) * K * c.sz : 0);
}

// global offset of interior point e (x fastest) of a patch
template <int DIM, int K>
__device__ __forceinline__ int64_t pv_interior(const PatchColour &c, int e)
{
  constexpr int M = 2 * K - 1;
  const int xi = e % M, yi = (e / M) % M, zi = DIM == 3 ? e / (M * M) : 0;
  return (xi + 1) + (yi + 1) * c.sy + (DIM == 3 ? (zi + 1) * c.sz : 0);
}

// r_I = b_I - scale A_ref x on the interior of each patch of the colour
// (A_ref = sum over directions of the patch stiffness in that direction
// times the patch mass in the others, reference cells)
template <int DIM, int K, typename T>
__global__ void __launch_bounds__(PVar<DIM, K>::NT)
    patch_residual_kernel(const T *__restrict__ x, const T *__restrict__ b, T *__restrict__ r,
                          const PatchColour c, T scale)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  using S = PVar<DIM, K>;
  constexpr int N1 = S::N1, M = S::M, NT = S::NT;
  const DegreeTables<K, T> &tb = c_tables<K, T>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T *Pm = reinterpret_cast<T *>(smem_raw), *Pl = Pm + N1 * N1, *X = Pl + N1 * N1;
  T *Z1 = X + S::BOX, *Z2 = Z1 + S::ZS, *V1 = Z2 + S::ZS, *V2 = V1 + S::VS;
  const int tid = threadIdx.x;
  const int64_t o = pv_origin<DIM, K>(c, blockIdx.x);
  for (int e = tid; e < N1 * N1; e += NT) {
    Pm[e] = tb.pmass[e];
    Pl[e] = tb.plap[e];
  }
  for (int e = tid; e < S::BOX; e += NT) {
    const int ex = e % N1, ey = (e / N1) % N1, ez = DIM == 3 ? e / (N1 * N1) : 0;
    X[e] = x[o + ex + ey * c.sy + (DIM == 3 ? ez * c.sz : 0)];
  }
  __syncthreads();
  if constexpr (DIM == 3) {
    // Z1 = M_z X, Z2 = L_z X on the interior z rows: [zi][y][x]
    for (int e = tid; e < S::ZS; e += NT) {
      const int zi = e / (N1 * N1), yx = e % (N1 * N1);
      T s1 = T(0), s2 = T(0);
      for (int z = 0; z < N1; ++z) {
        const T v = X[z * N1 * N1 + yx];
        s1 += Pm[(zi + 1) * N1 + z] * v;
        s2 += Pl[(zi + 1) * N1 + z] * v;
      }
      Z1[e] = s1;
      Z2[e] = s2;
    }
    __syncthreads();
    // V1 = M_y Z2 + L_y Z1, V2 = M_y Z1 on the interior y rows: [zi][yi][x]
    for (int e = tid; e < S::VS; e += NT) {
      const int zi = e / (M * N1), yi = (e / N1) % M, xx = e % N1;
      T s1 = T(0), s2 = T(0);
      for (int y = 0; y < N1; ++y) {
        const T z1 = Z1[zi * N1 * N1 + y * N1 + xx], z2 = Z2[zi * N1 * N1 + y * N1 + xx];
        s1 += Pm[(yi + 1) * N1 + y] * z2 + Pl[(yi + 1) * N1 + y] * z1;
        s2 += Pm[(yi + 1) * N1 + y] * z1;
      }
      V1[e] = s1;
      V2[e] = s2;
    }
    __syncthreads();
    // r = b - scale (M_x V1 + L_x V2) on the interior x rows
    for (int e = tid; e < S::INT; e += NT) {
      const int zi = e / (M * M), yi = (e / M) % M, xi = e % M;
      T s = T(0);
      for (int xx = 0; xx < N1; ++xx)
        s += Pm[(xi + 1) * N1 + xx] * V1[(zi * M + yi) * N1 + xx] + Pl[(xi + 1) * N1 + xx] * V2[(zi * M + yi) * N1 + xx];
      const int64_t g = o + pv_interior<DIM, K>(c, e);
      r[g] = b[g] - scale * s;
    }
  } else {
    // Z1 = M_y X, Z2 = L_y X on the interior y rows: [yi][x]
    for (int e = tid; e < S::ZS; e += NT) {
      const int yi = e / N1, xx = e % N1;
      T s1 = T(0), s2 = T(0);
      for (int y = 0; y < N1; ++y) {
        const T v = X[y * N1 + xx];
        s1 += Pm[(yi + 1) * N1 + y] * v;
        s2 += Pl[(yi + 1) * N1 + y] * v;
      }
      Z1[e] = s1;
      Z2[e] = s2;
    }
    __syncthreads();
    // r = b - scale (L_x Z1 + M_x Z2)
    for (int e = tid; e < S::INT; e += NT) {
      const int yi = e / M, xi = e % M;
      T s = T(0);
      for (int xx = 0; xx < N1; ++xx)
        s += Pl[(xi + 1) * N1 + xx] * Z1[yi * N1 + xx] + Pm[(xi + 1) * N1 + xx] * Z2[yi * N1 + xx];
      const int64_t g = o + pv_interior<DIM, K>(c, e);
      r[g] = b[g] - scale * s;
    }
  }
}

// out = Mat applied along axis `axis` (stride M^axis) of an M^DIM array;
// Mat(i, j) = Ev[j M + i] (S^T) if TRANSPOSE, else Ev[i M + j] (S)
template <int DIM, int K, typename T, bool TRANSPOSE>
__device__ __forceinline__ void pv_axis(const T *Ev, const T *in, T *out, int axis)
{
  constexpr int M = 2 * K - 1, INT = PVar<DIM, K>::INT, NT = PVar<DIM, K>::NT;
  const int st = axis == 0 ? 1 : axis == 1 ? M : M * M;
  for (int e = threadIdx.x; e < INT; e += NT) {
    const int i = (e / st) % M, base = e - i * st;
    T s = T(0);
    for (int j = 0; j < M; ++j) s += (TRANSPOSE ? Ev[j * M + i] : Ev[i * M + j]) * in[base + j * st];
    out[e] = s;
  }
  __syncthreads();
}

// x_I <- omega (x_I + inv_scale A_ref,II^{-1} r_I) for each patch of the
// colour: fast diagonalisation when inv is null, else the dense inverse
// `inv` (INT x INT, symmetric) of the reference-cell interior patch matrix
template <int DIM, int K, typename T>
__global__ void __launch_bounds__(PVar<DIM, K>::NT)
    patch_solve_kernel(T *__restrict__ x, const T *__restrict__ r, const T *__restrict__ inv,
                       const PatchColour c, T omega, T inv_scale)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  using S = PVar<DIM, K>;
  constexpr int M = S::M, NT = S::NT, INT = S::INT;
  const DegreeTables<K, T> &tb = c_tables<K, T>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T *Ev = reinterpret_cast<T *>(smem_raw), *Lm = Ev + M * M, *Q0 = Lm + M, *Q1 = Q0 + INT;
  const int tid = threadIdx.x;
  const int64_t o = pv_origin<DIM, K>(c, blockIdx.x);
  for (int e = tid; e < M * M; e += NT) Ev[e] = tb.evec[e];
  for (int e = tid; e < M; e += NT) Lm[e] = tb.eval[e];
  for (int e = tid; e < INT; e += NT) Q0[e] = r[o + pv_interior<DIM, K>(c, e)];
  __syncthreads();
  const T *sol;
  if (inv) {
    for (int e = tid; e < INT; e += NT) {
      T s = T(0);
      for (int j = 0; j < INT; ++j) s += inv[static_cast<int64_t>(j) * INT + e] * Q0[j];
      Q1[e] = s;
    }
    __syncthreads();
    sol = Q1;
  } else {
    // S^T along every axis, 1 / (sum of eigenvalues), S along every axis
    T *a = Q0, *bq = Q1;
    for (int ax = 0; ax < DIM; ++ax) {
      pv_axis<DIM, K, T, true>(Ev, a, bq, ax);
      T *t = a;
      a = bq;
      bq = t;
    }
    for (int e = tid; e < INT; e += NT) {
      const int xi = e % M, yi = (e / M) % M, zi = DIM == 3 ? e / (M * M) : 0;
      a[e] /= Lm[xi] + Lm[yi] + (DIM == 3 ? Lm[zi] : T(0));
    }
    __syncthreads();
    for (int ax = DIM - 1; ax >= 0; --ax) {
      pv_axis<DIM, K, T, false>(Ev, a, bq, ax);
      T *t = a;
      a = bq;
      bq = t;
    }
    sol = a;
  }
  for (int e = tid; e < INT; e += NT) {
    const int64_t g = o + pv_interior<DIM, K>(c, e);
    x[g] = omega * (x[g] + inv_scale * sol[e]);
  }
}

// x += w a over n entries (the additive step's damped correction)
template <typename T>
__global__ void scaled_add_kernel(T *__restrict__ x, const T *__restrict__ a, T w, int64_t n)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    x[i] += w * a[i];
}

}  // namespace tps
