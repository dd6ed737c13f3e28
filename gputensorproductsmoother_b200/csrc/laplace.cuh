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
  extern __shared__ __align__(16) unsigned char smem_raw[];
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

// ---------------------------------------------------------------------------
// 3D operator, z-streaming form.  A CTA owns TX x TY cells in x, y and marches
// through a range of cell layers in z.  Each input plane (with a one-cell xy
// halo) is contracted once in x (M, L) and once in y, giving the planes
// T1 = M_y M_x u and T2 = (L_y M_x + M_y L_x) u of the output tile; the z
// direction is then applied cell by cell: for cell layer c the (k+1)x(k+1)
// cell matrices act on the k+1 planes ck..(c+1)k of T1 (stiffness) and T2
// (mass), the k+1 results go to planes ck..(c+1)k, and the last one -- the
// vertex plane shared with cell c+1 -- is carried in a register to the next
// layer.  A CTA starts one layer early to form the carry of its first plane,
// so every input plane is read from memory about (1 + 1/CZ) times in z (xy
// halo: ((T+1)k+1)^2/(Tk)^2) instead of the brick kernel's full halo in all
// three directions.  The next layer's k input planes are loaded into
// registers while the current layer is contracted; each thread's staged xy
// offsets are computed once, so a prefetched entry costs one add and a load.
// CTAs per SM the register budget must allow: two (at most 128 registers for
// 256 threads), which doubles the resident warps of this latency-bound kernel
// (measured on B200, ms per apply, one CTA vs two: Q4 64^3 FP64 0.255 vs
// 0.198, FP32 0.136 vs 0.131; Q3 32^3 FP64 0.038 vs 0.024; Q7 32^3 FP64 0.321
// vs 0.296), except Q7 FP32, which spills 444 bytes under the cap (0.169 vs
// 0.388 ms) and keeps one
template <int K, typename T>
constexpr int opstream_minb()
{
#ifdef TPS_OPSTREAM_MINB
  return TPS_OPSTREAM_MINB(K);
#else
  return (K == 7 && sizeof(T) == 4) ? 1 : 2;
#endif
}
template <int K, typename T>
struct OpStream {
  static constexpr int TX = K == 1 ? 16 : K == 2 ? 8 : K <= 4 ? 4 : K == 5 ? 3 : 2, TY = TX;  // cells per CTA in x, y
  static constexpr int OX = TX * K, OY = TY * K;      // output tile
  static constexpr int WX = (TX + 1) * K + 1, WY = (TY + 1) * K + 1;  // staged plane
  static constexpr int NT = (OX * OY + 31) / 32 * 32;
  static constexpr int CZ = 8;                        // cell layers per CTA (at most; see opstream_layers)
  static constexpr int PL = WX * WY;                  // one staged input plane
  static constexpr int XS = WY * OX;                  // one x-contracted plane (per product)
  static constexpr int TS = OY * OX;                  // one xy-contracted plane (per product)
  // shared memory (elements): IN[K][PL] | X1[K][XS] | X2[K][XS] | T1[K+1][TS] | T2[K+1][TS]
  static constexpr int OFF_X1 = K * PL, OFF_X2 = OFF_X1 + K * XS, OFF_T1 = OFF_X2 + K * XS;
  static constexpr int OFF_T2 = OFF_T1 + (K + 1) * TS;
  static constexpr int ELEMS = OFF_T2 + (K + 1) * TS;
  static constexpr int EPT = (PL + NT - 1) / NT;      // staged xy entries per thread and plane
  static constexpr int MINB = opstream_minb<K, T>();   // CTAs per SM the registers must allow
};

// cell layers per CTA for a level of n cells per direction: the most (up to
// CZ, fewer leading layers recomputed) that still gives at least `want` CTAs;
// one on small levels, where a CTA's layer march is the latency
template <int K, typename T>
inline int opstream_layers(int n, int want)
{
  using S = OpStream<K, T>;
  const int xy = ((n + S::TX - 1) / S::TX) * ((n + S::TY - 1) / S::TY);
  for (int cz = S::CZ; cz > 1; cz /= 2)
    if (xy * ((n + cz - 1) / cz) >= want) return cz;
  return 1;
}

template <int K, typename T, OpMode MODE>
__global__ void __launch_bounds__(OpStream<K, T>::NT, OpStream<K, T>::MINB)
    laplace3d_stream_kernel(T *__restrict__ dst, const T *__restrict__ src, const T *__restrict__ rhs,
                            int N1g, int n_cells, int64_t sy, int64_t sz, T scale, int cz)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  using S = OpStream<K, T>;
  constexpr int NT = S::NT, WX = S::WX, WY = S::WY, OX = S::OX, OY = S::OY, PL = S::PL;
  constexpr int XS = S::XS, TS = S::TS, EPT = S::EPT;
  const DegreeTables<K, T> &tb = c_tables<K, T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sm = reinterpret_cast<T *>(smem_raw);
  T *IN = sm, *X1 = sm + S::OFF_X1, *X2 = sm + S::OFF_X2, *T1 = sm + S::OFF_T1, *T2 = sm + S::OFF_T2;
  const int tid = threadIdx.x;
  const int cx0 = blockIdx.x * S::TX, cy0 = blockIdx.y * S::TY;
  const int gx0 = (cx0 - 1) * K, gy0 = (cy0 - 1) * K;  // staged plane origin
  const int cz_begin = blockIdx.z * cz;  // cz cell layers per CTA
  const int cz_end = min(cz_begin + cz, n_cells);
  const int c_first = cz_begin > 0 ? cz_begin - 1 : 0;  // leading layer: carry only

  // this thread's staged xy entries (fixed for every plane): global xy offset
  // and whether the entry lies in the mesh
  int64_t xoff[EPT];
  bool xok[EPT];
#pragma unroll
  for (int j = 0; j < EPT; ++j) {
    const int l = tid + j * NT, lx = l % WX, ly = l / WX;
    const int gx = gx0 + lx, gy = gy0 + ly;
    xok[j] = l < PL && gx >= 0 && gx < N1g && gy >= 0 && gy < N1g;
    xoff[j] = xok[j] ? gx + gy * sy : 0;
  }
  // load planes z0 .. z0+np-1 (np <= K) of the staged tile into registers
  T pre[K][EPT];
  auto prefetch = [&](int z0, int np) {
#pragma unroll
    for (int p = 0; p < K; ++p) {
      const int gz = z0 + p;
      const bool zok = p < np && gz >= 0 && gz < N1g;
#pragma unroll
      for (int j = 0; j < EPT; ++j) pre[p][j] = (zok && xok[j]) ? __ldg(&src[xoff[j] + gz * sz]) : T(0);
    }
  };
  auto commit = [&]() {
#pragma unroll
    for (int p = 0; p < K; ++p)
#pragma unroll
      for (int j = 0; j < EPT; ++j) {
        const int l = tid + j * NT;
        if (l < PL) IN[p * PL + l] = pre[p][j];
      }
  };
  // x then y contraction of staged planes 0..np-1 into T slots slot0.. (mod K+1)
  auto contract_xy = [&](int np, int slot0) {
    for (int t = tid; t < np * WY * S::TX; t += NT) {
      const int c = t % S::TX, r = t / S::TX;  // r = p * WY + y
      const T *s = IN + (r / WY) * PL + (r % WY) * WX + c * K;
      T v[2 * K + 1], o1[K], o2[K];
#pragma unroll
      for (int j = 0; j <= 2 * K; ++j) v[j] = s[j];
      band_apply<K, T>(tb.cmass, v, o1);
      band_apply<K, T>(tb.clap, v, o2);
      T *d1 = X1 + r * OX + c * K, *d2 = X2 + r * OX + c * K;
#pragma unroll
      for (int a = 0; a < K; ++a) {
        d1[a] = o1[a];
        d2[a] = o2[a];
      }
    }
    __syncthreads();
    for (int t = tid; t < np * OX * S::TY; t += NT) {
      const int xo = t % OX, r = t / OX;  // r = p * TY + cell row
      const int p = r / S::TY, c = r % S::TY;
      const T *s1 = X1 + p * XS + c * K * OX + xo, *s2 = X2 + p * XS + c * K * OX + xo;
      T v1[2 * K + 1], v2[2 * K + 1], o1[K], o2[K], o3[K];
#pragma unroll
      for (int j = 0; j <= 2 * K; ++j) {
        v1[j] = s1[j * OX];
        v2[j] = s2[j * OX];
      }
      band_apply<K, T>(tb.cmass, v1, o1);
      band_apply<K, T>(tb.clap, v1, o2);
      band_apply<K, T>(tb.cmass, v2, o3);
      const int slot = (slot0 + p) % (K + 1);
      T *d1 = T1 + slot * TS + c * K * OX + xo, *d2 = T2 + slot * TS + c * K * OX + xo;
#pragma unroll
      for (int a = 0; a < K; ++a) {
        d1[a * OX] = o1[a];
        d2[a * OX] = o2[a] + o3[a];
      }
    }
    __syncthreads();
  };

  // prime: plane c_first*K into slot 0
  int base = 0;  // slot of plane c*K
  prefetch(c_first * K, 1);
  commit();
  __syncthreads();
  contract_xy(1, base);
  prefetch(c_first * K + 1, K);  // the first layer's new planes
  const int tx = tid % OX, ty = tid / OX;
  const bool owner = tid < OX * OY;
  const int gx = cx0 * K + tx, gy = cy0 * K + ty;
  const bool xy_in = owner && gx > 0 && gx < N1g - 1 && gy > 0 && gy < N1g - 1;
  T carry = T(0);
  for (int c = c_first; c < cz_end; ++c) {
    commit();
    __syncthreads();
    if (c + 1 < cz_end) prefetch((c + 1) * K + 1, K);  // next layer, overlapped with the contractions
    contract_xy(K, base + 1);
    // z: cell matrices on planes cK..(c+1)K
    if (owner) {
      T u1[K + 1], u2[K + 1];
#pragma unroll
      for (int b = 0; b <= K; ++b) {
        const int slot = (base + b) % (K + 1);
        u1[b] = T1[slot * TS + ty * OX + tx];
        u2[b] = T2[slot * TS + ty * OX + tx];
      }
      T out[K + 1];
#pragma unroll
      for (int a = 0; a <= K; ++a) {
        T acc = T(0);
#pragma unroll
        for (int b = 0; b <= K; ++b) acc += tb.clap[a * (K + 1) + b] * u1[b] + tb.cmass[a * (K + 1) + b] * u2[b];
        out[a] = acc;
      }
      out[0] += carry;
      carry = out[K];
      if (c >= cz_begin && xy_in) {
#pragma unroll
        for (int a = 0; a < K; ++a) {
          const int gz = c * K + a;
          if (gz < 1 || gz > N1g - 2) continue;
          const int64_t gi = gx + gy * sy + gz * sz;
          const T val = scale * out[a];
          if constexpr (MODE == OpMode::Vmult)
            dst[gi] = val;
          else
            dst[gi] = rhs[gi] - val;
        }
      }
    }
    base = (base + K) % (K + 1);
    __syncthreads();  // the T slots of this layer's first planes are refilled next
  }
}

}  // namespace tps
