// Matrix-free Laplace operator on a uniform Cartesian Q_k level, sm_100a.
//
// Reference behaviour: LaplaceOperator::vmult (include/laplace_operator.cuh:86-101)
// = cell loop of the gradient form with QGauss(k+1)
// (include/dealii/cuda_mf.template.cuh:532-563, include/dealii/cuda_fee.cuh:273-529)
// scattered with atomicAdd, then dst = src on the Dirichlet rows
// (include/dealii/cuda_mf.template.cuh:492-508).
//
// B200 design: on a uniform tensor mesh with exact Gauss integration the
// assembled operator is the Kronecker sum of the global 1D mass/stiffness
// matrices, A = s * (L_z M_y M_x + M_z L_y M_x + M_z M_y L_x), s = h^(dim-2).
// Each CTA owns a brick of cells, stages the brick plus a one-cell halo in
// shared memory and applies five banded 1D contractions (interior outputs
// only) -- a gather with no atomics, hence deterministic, at ~42 multiply-adds
// per DoF instead of the ~175 of the cell-wise sum factorization.  A global 1D
// row of node c*k+a couples to the k+1 nodes of cell c, plus (a == 0) the k+1
// nodes of cell c-1; one thread computes the k outputs of one cell segment
// from 2k+1 register-resident inputs, so every coefficient is a compile-time
// constant-bank operand.
#pragma once

#include "tps_common.cuh"

namespace tps {

enum class OpMode { Vmult = 0, Residual = 1 };

template <int DIM, int K>
struct OpTile {
  // cells per CTA in x, y, z
  static constexpr int CX = DIM == 3 ? (K == 1 ? 8 : K <= 4 ? 4 : 2) : (K == 1 ? 32 : K == 2 ? 16 : 8);
  static constexpr int CY = DIM == 3 ? (K == 1 ? 8 : K == 2 ? 4 : K <= 5 ? 2 : K == 6 ? 2 : 1)
                                     : (K <= 4 ? 8 : 4);
  static constexpr int CZ = DIM == 3 ? (K == 1 ? 8 : K == 2 ? 4 : K <= 5 ? 2 : 1) : 1;
  static constexpr int WX = (CX + 1) * K + 1;  // staged input extents
  static constexpr int WY = (CY + 1) * K + 1;
  static constexpr int WZ = DIM == 3 ? (CZ + 1) * K + 1 : 1;
  static constexpr int OX = CX * K, OY = CY * K, OZ = DIM == 3 ? CZ * K : 1;  // outputs
  static constexpr int IN = WX * WY * WZ;
  // contracted arrays store x permuted, x' = a*CX + c for node c*K+a of the
  // tile, in rows of RX >= OX entries: consecutive threads (consecutive c)
  // then touch consecutive shared-memory words
  static constexpr int RX = OX + CX;
  static constexpr int TS = WZ * WY * RX;          // one x-contracted array
  static constexpr int US = DIM == 3 ? WZ * OY * RX : 0;  // one xy-contracted array
  // U1/U2 reuse the input region once the x stage is done
  static constexpr int REGION0 = IN > 2 * US ? IN : 2 * US;
  static constexpr int SMEM_ELEMS = REGION0 + 2 * TS;
  static constexpr int NT = 256;
};

// k outputs of one cell segment of a global 1D banded product:
// v[0..2k] = values at nodes (c-1)k .. (c+1)k; out[a] = row c*k+a.
template <int K, typename T>
__device__ __forceinline__ void band_apply(const T *mat /* (k+1)^2 cell matrix */,
                                           const T (&v)[2 * K + 1], T (&out)[K])
{
#pragma unroll
  for (int a = 0; a < K; ++a) {
    T s = T(0);
#pragma unroll
    for (int b = 0; b <= K; ++b) s += mat[a * (K + 1) + b] * v[K + b];
    if (a == 0) {
#pragma unroll
      for (int b = 0; b <= K; ++b) s += mat[K * (K + 1) + b] * v[b];
    }
    out[a] = s;
  }
}

template <int DIM, int K, typename T, OpMode MODE>
__global__ void __launch_bounds__(OpTile<DIM, K>::NT, 2)
    laplace_kernel(T *__restrict__ dst, const T *__restrict__ src, const T *__restrict__ rhs,
                   int N1g, int64_t sy, int64_t sz, T scale)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  using Tl = OpTile<DIM, K>;
  constexpr int NT = Tl::NT, WX = Tl::WX, WY = Tl::WY, WZ = Tl::WZ;
  constexpr int OX = Tl::OX, OY = Tl::OY, OZ = Tl::OZ, RX = Tl::RX;
  const DegreeTables<K, T> &tb = c_tables<K, T>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T *sIn = reinterpret_cast<T *>(smem_raw);
  T *U1 = sIn, *U2 = sIn + Tl::US;
  T *T1 = sIn + Tl::REGION0, *T2 = T1 + Tl::TS;

  const int cx0 = blockIdx.x * Tl::CX, cy0 = blockIdx.y * Tl::CY, cz0 = blockIdx.z * Tl::CZ;
  const int gx0 = cx0 * K, gy0 = cy0 * K, gz0 = DIM == 3 ? cz0 * K : 0;
  // stage 0: input brick with a one-cell halo (zero outside the mesh); the
  // loop has a compile-time trip count and is unrolled in chunks so that
  // every thread keeps a chunk of independent loads in flight
  constexpr int NLOAD = (Tl::IN + NT - 1) / NT;
  constexpr int CH = NLOAD < 8 ? NLOAD : 8;
#pragma unroll 1
  for (int i0 = 0; i0 < NLOAD; i0 += CH) {
    T v[CH];
#pragma unroll
    for (int c = 0; c < CH; ++c) {
      const int e = threadIdx.x + (i0 + c) * NT;
      const int lx = e % WX, ly = (e / WX) % WY, lz = DIM == 3 ? e / (WX * WY) : 0;
      const int gx = gx0 - K + lx, gy = gy0 - K + ly, gz = DIM == 3 ? gz0 - K + lz : 0;
      v[c] = T(0);
      if (i0 + c < NLOAD && e < Tl::IN && gx >= 0 && gx < N1g && gy >= 0 && gy < N1g &&
          (DIM == 2 || (gz >= 0 && gz < N1g)))
        v[c] = __ldg(&src[gx + gy * sy + gz * sz]);
    }
#pragma unroll
    for (int c = 0; c < CH; ++c) {
      const int e = threadIdx.x + (i0 + c) * NT;
      if (i0 + c < NLOAD && e < Tl::IN) sIn[e] = v[c];
    }
  }
  __syncthreads();

  // stage x: T1 = M_x in, T2 = L_x in  (all staged y,z; output x in [0,OX))
  for (int t = threadIdx.x; t < WZ * WY * Tl::CX; t += NT) {
    const int c = t % Tl::CX, line = t / Tl::CX;
    const T *s = sIn + line * WX + c * K;
    T v[2 * K + 1], o1[K], o2[K];
#pragma unroll
    for (int j = 0; j <= 2 * K; ++j) v[j] = s[j];
    band_apply<K, T>(tb.cmass, v, o1);
    band_apply<K, T>(tb.clap, v, o2);
    T *d1 = T1 + line * RX + c, *d2 = T2 + line * RX + c;
#pragma unroll
    for (int a = 0; a < K; ++a) {
      d1[a * Tl::CX] = o1[a];
      d2[a * Tl::CX] = o2[a];
    }
  }
  __syncthreads();

  if constexpr (DIM == 2) {
    // stage y: out = s (L_y T1 + M_y T2)
    for (int t = threadIdx.x; t < OX * Tl::CY; t += NT) {
      const int xp = t % OX, c = t / OX;  // xp: permuted x
      T v1[2 * K + 1], v2[2 * K + 1], o1[K], o2[K];
#pragma unroll
      for (int j = 0; j <= 2 * K; ++j) {
        v1[j] = T1[(c * K + j) * RX + xp];
        v2[j] = T2[(c * K + j) * RX + xp];
      }
      band_apply<K, T>(tb.clap, v1, o1);
      band_apply<K, T>(tb.cmass, v2, o2);
      const int gx = gx0 + (xp % Tl::CX) * K + xp / Tl::CX;
      if (gx < 1 || gx > N1g - 2) continue;
#pragma unroll
      for (int a = 0; a < K; ++a) {
        const int gy = gy0 + c * K + a;
        if (gy < 1 || gy > N1g - 2) continue;
        const int64_t gi = gx + gy * sy;
        const T val = scale * (o1[a] + o2[a]);
        if constexpr (MODE == OpMode::Vmult)
          dst[gi] = val;
        else
          dst[gi] = rhs[gi] - val;
      }
    }
  } else {
    // stage y: U1 = M_y T1, U2 = L_y T1 + M_y T2
    for (int t = threadIdx.x; t < WZ * OX * Tl::CY; t += NT) {
      const int xp = t % OX, r = t / OX;
      const int c = r % Tl::CY, z = r / Tl::CY;
      T v1[2 * K + 1], v2[2 * K + 1], o1[K], o2[K], o3[K];
#pragma unroll
      for (int j = 0; j <= 2 * K; ++j) {
        v1[j] = T1[(z * WY + c * K + j) * RX + xp];
        v2[j] = T2[(z * WY + c * K + j) * RX + xp];
      }
      band_apply<K, T>(tb.cmass, v1, o1);
      band_apply<K, T>(tb.clap, v1, o2);
      band_apply<K, T>(tb.cmass, v2, o3);
#pragma unroll
      for (int a = 0; a < K; ++a) {
        U1[(z * OY + c * K + a) * RX + xp] = o1[a];
        U2[(z * OY + c * K + a) * RX + xp] = o2[a] + o3[a];
      }
    }
    __syncthreads();
    // stage z: out = s (L_z U1 + M_z U2)
    for (int t = threadIdx.x; t < OY * OX * Tl::CZ; t += NT) {
      const int yx = t % (OY * OX), c = t / (OY * OX);
      const int xp = yx % OX, yy = yx / OX;
      T v1[2 * K + 1], v2[2 * K + 1], o1[K], o2[K];
#pragma unroll
      for (int j = 0; j <= 2 * K; ++j) {
        v1[j] = U1[((c * K + j) * OY + yy) * RX + xp];
        v2[j] = U2[((c * K + j) * OY + yy) * RX + xp];
      }
      band_apply<K, T>(tb.clap, v1, o1);
      band_apply<K, T>(tb.cmass, v2, o2);
      const int gx = gx0 + (xp % Tl::CX) * K + xp / Tl::CX, gy = gy0 + yy;
      if (gx < 1 || gx > N1g - 2 || gy < 1 || gy > N1g - 2) continue;
#pragma unroll
      for (int a = 0; a < K; ++a) {
        const int gz = gz0 + c * K + a;
        if (gz < 1 || gz > N1g - 2) continue;
        const int64_t gi = gx + gy * sy + gz * sz;
        const T val = scale * (o1[a] + o2[a]);
        if constexpr (MODE == OpMode::Vmult)
          dst[gi] = val;
        else
          dst[gi] = rhs[gi] - val;
      }
    }
  }
  (void)OZ;
}

}  // namespace tps
