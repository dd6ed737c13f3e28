// Shared device-side definitions: per-degree 1D tables in __constant__
// memory, level geometry, and launch helpers.
//
// Design note (B200): every 1D table is level-independent (mesh-size factors
// are applied as scalars), so one copy per (degree, precision) lives in
// constant memory.  Contraction loops are fully unrolled over compile-time
// degrees, so each coefficient becomes an immediate constant-bank operand of
// the FMA: no shared-memory or register traffic for the matrices.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "launch.cuh"

namespace tps {

template <int K>
struct Dims {
  static constexpr int NP = K + 1;      // DoFs per cell and direction
  static constexpr int N1 = 2 * K + 1;  // DoFs per patch and direction
  static constexpr int M = 2 * K - 1;   // interior DoFs per patch and direction
};

// Two values processed by one instruction: packed FP32x2 arithmetic on sm_100
// (__ffma2_rn), component-wise FP64.
template <typename T>
struct Pair;
template <>
struct Pair<float> {
  using type = float2;
  static __host__ __device__ __forceinline__ float2 make(float a, float b) { return make_float2(a, b); }
  static __device__ __forceinline__ float2 fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
};
template <>
struct Pair<double> {
  using type = double2;
  static __host__ __device__ __forceinline__ double2 make(double a, double b) { return make_double2(a, b); }
  static __device__ __forceinline__ double2 fma(double2 a, double2 b, double2 c)
  {
    return make_double2(::fma(a.x, b.x, c.x), ::fma(a.y, b.y, c.y));
  }
};

// a * b + c as one fused multiply-add in either precision: written out where
// the sum of two products would otherwise leave the choice of the fused
// product to the compiler, so that kernels of different shapes round alike
__device__ __forceinline__ float fmadd(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmadd(double a, double b, double c) { return __fma_rn(a, b, c); }
// a + b and a - b that the compiler may not fuse with a product operand
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

template <int K, typename T>
struct DegreeTables {
  T pmass[Dims<K>::N1 * Dims<K>::N1];   // patch mass (reference cells)
  T plap[Dims<K>::N1 * Dims<K>::N1];    // patch stiffness (reference cells)
  T cmass[Dims<K>::NP * Dims<K>::NP];   // cell mass
  T clap[Dims<K>::NP * Dims<K>::NP];    // cell stiffness
  T evec[Dims<K>::M * Dims<K>::M];      // interior eigenvectors (columns)
  T eval[Dims<K>::M];                   // interior eigenvalues (reference scaling)
  T prol[Dims<K>::N1 * Dims<K>::NP];    // 1D prolongation (child node x coarse basis)
  T qwshape[Dims<K>::NP * Dims<K>::NP]; // QGauss(k+1) weight times basis: w_q phi_i(x_q), [q][i]
  // even/odd folded interior rows of the centro-symmetric patch matrices A:
  // row r < k-1 (A row r+1, paired with row 2k-1-r):
  //   fe[r][j] = (A[r+1][j] + A[r+1][2k-j])/2 (j < k), fe[r][k] = A[r+1][k]
  //   fo[r][j] = (A[r+1][j] - A[r+1][2k-j])/2 (j < k)
  // row k-1 is the centre row A[k][.] (fe only)
  T pmass_fe[K * (K + 1)];
  T plap_fe[K * (K + 1)];
  T pmass_fo[K > 1 ? (K - 1) * K : 1];
  T plap_fo[K > 1 ? (K - 1) * K : 1];
  // the same folded rows as (even, odd) coefficient pairs {fe[r][j], fo[r][j]}, r < k-1, j < k
  typename Pair<T>::type pmass_fp[K > 1 ? (K - 1) * K : 1];
  typename Pair<T>::type plap_fp[K > 1 ? (K - 1) * K : 1];
  // eigenvector pairs {S[r][q], S[r][k+q]} for r, q < k-1 (even mode q, odd mode k+q)
  typename Pair<T>::type evec_p[K > 1 ? (K - 1) * (K - 1) : 1];
};


template <int K, typename T>
__constant__ DegreeTables<K, T> c_tables;

// Geometry of one level: n cells per direction, N1 = n*k+1 DoFs per direction.
struct LevelGeom {
  int n;       // cells per direction
  int N1;      // DoFs per direction
  int64_t N;   // total DoFs
  double h;    // cell size 1/n
};

inline unsigned ceil_div(int64_t a, int64_t b) { return static_cast<unsigned>((a + b - 1) / b); }

}  // namespace tps
