// 3D fused vertex-patch smoother, one launch per colour (sm_100a).
//
// Reference behaviour: LevelVertexPatch::patch_loop_fused with
// loop_kernel_fused_cf + LocalSmoother<FUSED_CF> (include/loop_kernel.cuh:962-1060,
// include/evaluate_kernel.cuh:501-590, 1327-1434, 2058-2163): for every patch p
// of the colour,  x_I(p) <- omega (x_I(p) + A_II^{-1} (b - A_p x)_I).
//
// Algebra used here: with x = x_I + x_B on the patch box,
//     omega (x_I + A_II^{-1}(b_I - A_II x_I - A_IB x_B)) = omega A_II^{-1}(b_I - A_IB x_B),
// so the old interior values are never needed (the idea of the reference's
// FUSED_BD variant, include/loop_kernel.cuh:667-783): the box residual is
// evaluated with the interior of x set to zero, which turns the interior
// z-lines of the first contraction into two-term lines.
//
// B200 design:
//  * persistent CTAs; each CTA walks batches of PPB patches of the colour;
//  * the (2k+1)^3 box of x and the (2k-1)^2 x W slab of b of every patch of
//    the next batch are fetched by TMA (cp.async.bulk.tensor.3d) into a second
//    shared-memory stage while the current batch is computed; completion is
//    tracked by one mbarrier per stage with a bounded wait;
//  * contractions: z (M, L) -> y (3 products) -> x (2 products) + S^T_x ->
//    S^T_y -> S^T_z, scale, S_z -> S_x -> S_y + store.  Every contraction keeps
//    one 1D line per thread in registers and applies the centro-symmetric 1D
//    matrices in even/odd folded form (about half the dense multiply-adds)
//    with scalar FMAs whose coefficients are constant-bank operands (degree
//    <= 5), or in a packed form (__ffma2_rn on (even, odd) pairs; degree >= 6,
//    where it measured faster; see sm3_packed).  The
//    sums of two products (M_y Z2 + L_y Z1, M_x V1 + L_x V2) run as one
//    accumulation chain, and every kernel variant uses the same chains, so
//    the variants give bit-identical sweeps;
//  * per-batch patch offsets are computed once into shared memory; the
//    thread count matches the widest stage (the y stage), and the cheap
//    interior z-lines are processed two per thread;
//  * a second loader variant (plain coalesced loads) serves vectors whose
//    pitch is not 16-byte aligned (the C-ABI level operations on caller
//    vectors); the compute path is shared.
#pragma once

#include <cuda.h>

#include "intdiv.cuh"
#include "ptx.cuh"
#include "tps_common.cuh"

namespace tps {

// default patches per CTA batch: enough lines per stage, two to three CTAs per SM
template <int K, typename T>
constexpr int sm3_default_ppb()
{
  return sizeof(T) == 4 ? (K == 1 ? 32 : K == 2 ? 16 : K == 3 ? 8 : K == 4 ? 4 : K <= 6 ? 2 : 1)
                        : (K == 1 ? 16 : K == 2 ? 8 : K == 3 ? 4 : K == 4 ? 2 : 1);
}

template <int K, typename T, int PPB_ = 0>
struct Sm3 {
  static constexpr int N1 = 2 * K + 1, M = 2 * K - 1;
  static constexpr int A = 16 / static_cast<int>(sizeof(T));  // TMA x-alignment (elements)
  static constexpr int W = ((N1 + A - 1) + A - 1) / A * A;    // staged row width
  static constexpr int XBOX = N1 * N1 * W;
  static constexpr int BBOX = M * M * W;
  static constexpr int ALIGN = 128 / static_cast<int>(sizeof(T));  // TMA destinations: 128 B
  static constexpr int ZSZ = M * N1 * N1;  // z-contracted  [zi][y][x]
  static constexpr int VSZ = M * M * N1;   // zy-contracted [zi][yi][x]
  static constexpr int QSZ = M * M * M;
  // the x box region also holds V1/V2 once the z stage is done
  static constexpr int XREG = XBOX > 2 * VSZ ? XBOX : 2 * VSZ;
  static constexpr int BOFF = (XREG + ALIGN - 1) / ALIGN * ALIGN;    // b slab inside a stage
  static constexpr int STAGE = (BOFF + BBOX + ALIGN - 1) / ALIGN * ALIGN;  // per patch
  static constexpr int RING = N1 * N1 - M * M;  // boundary lines of a z-face
  static constexpr int IPAIR = (M * M + 1) / 2;  // interior z-lines, two per task
  // patches per batch (PPB_ = 0: the default; the autotuner picks among variants)
  static constexpr int PPB = PPB_ > 0 ? PPB_ : sm3_default_ppb<K, T>();
  // threads = widest stage (y lines), rounded to warps
  static constexpr int NT_RAW = (PPB * M * N1 + 31) / 32 * 32;
  static constexpr int NT = NT_RAW < 64 ? 64 : NT_RAW;
  // shared memory layout (elements of T): 2 stages | Z1 | Z2 | 1/(lambda sums)
  static constexpr int OFF_Z1 = 2 * PPB * STAGE;
  static constexpr int OFF_Z2 = OFF_Z1 + PPB * ZSZ;
  static constexpr int OFF_RL = OFF_Z2 + PPB * ZSZ;
  static constexpr int ELEMS = (OFF_RL + QSZ + ALIGN - 1) / ALIGN * ALIGN;
  // tail: two mbarriers, the wait flag, per-batch patch offsets
  static constexpr size_t TAIL_BAR = sizeof(T) * ELEMS;
  static constexpr size_t TAIL_BASE = TAIL_BAR + 32;
  static constexpr size_t TAIL_XO = TAIL_BASE + 8 * PPB;
  static constexpr size_t BYTES = TAIL_XO + 4 * PPB + 16;
};

// v (2k+1 values) -> (e_j, o_j) pairs, j < k, and the centre e_k
template <int K, typename T>
__device__ __forceinline__ void fold_pairs(const T (&v)[2 * K + 1],
                                           typename Pair<T>::type (&eo)[K > 1 ? K : 1], T &ec)
{
#pragma unroll
  for (int j = 0; j < K; ++j) eo[j] = Pair<T>::make(v[j] + v[2 * K - j], v[j] - v[2 * K - j]);
  ec = v[K];
}

// interior rows 1..2k-1 of A v for a centro-symmetric (2k+1)^2 patch matrix
// from the folded input; the even/odd partial sums of the output pair
// (r, 2k-2-r) share one packed accumulator
template <int K, typename T>
__device__ __forceinline__ void fold_rows2(const typename Pair<T>::type *fp, const T *fe,
                                           const typename Pair<T>::type (&eo)[K > 1 ? K : 1],
                                           const T ec, T (&out)[2 * K - 1])
{
  using P = Pair<T>;
  constexpr int M = 2 * K - 1;
#pragma unroll
  for (int r = 0; r < K - 1; ++r) {
    typename P::type acc = P::make(fe[r * (K + 1) + K] * ec, T(0));
#pragma unroll
    for (int j = 0; j < K; ++j) acc = P::fma(fp[r * K + j], eo[j], acc);
    out[r] = acc.x + acc.y;
    out[M - 1 - r] = acc.x - acc.y;
  }
  T sc = fe[(K - 1) * (K + 1) + K] * ec;
#pragma unroll
  for (int j = 0; j < K; ++j) sc += fe[(K - 1) * (K + 1) + j] * (eo[j].x);
  out[K - 1] = sc;
}

// The same rows with scalar FMAs: every coefficient is a constant-bank
// operand of its FMA (the packed pairs above need a constant load per pair).
// Every chain starts with a product and continues with explicit fused
// multiply-adds in a fixed order, so the rounding does not depend on which
// product the compiler would fuse (the packed-pair kernel repeats it exactly).
template <int K, typename T>
__device__ __forceinline__ void fold_rows_s(const T *fe, const T *fo, const typename Pair<T>::type (&eo)[K > 1 ? K : 1],
                                            const T ec, T (&out)[2 * K - 1])
{
  constexpr int M = 2 * K - 1;
#pragma unroll
  for (int r = 0; r < K - 1; ++r) {
    T e = fe[r * (K + 1) + K] * ec, o = fo[r * K] * eo[0].y;
    e = fmadd(fe[r * (K + 1)], eo[0].x, e);
#pragma unroll
    for (int j = 1; j < K; ++j) {
      e = fmadd(fe[r * (K + 1) + j], eo[j].x, e);
      o = fmadd(fo[r * K + j], eo[j].y, o);
    }
    out[r] = add_rn(e, o);
    out[M - 1 - r] = sub_rn(e, o);
  }
  T sc = fe[(K - 1) * (K + 1) + K] * ec;
#pragma unroll
  for (int j = 0; j < K; ++j) sc = fmadd(fe[(K - 1) * (K + 1) + j], eo[j].x, sc);
  out[K - 1] = sc;
}

// interior rows of A u + B v for two centro-symmetric patch matrices from
// folded inputs: one accumulation chain per even/odd partial sum, so the sum
// costs no more combining adds than a single product
template <int K, typename T>
__device__ __forceinline__ void fold_rows_sum_s(const T *fea, const T *foa,
                                                const typename Pair<T>::type (&eoa)[K > 1 ? K : 1], const T eca,
                                                const T *feb, const T *fob,
                                                const typename Pair<T>::type (&eob)[K > 1 ? K : 1], const T ecb,
                                                T (&out)[2 * K - 1])
{
  constexpr int M = 2 * K - 1;
#pragma unroll
  for (int r = 0; r < K - 1; ++r) {
    T e = fea[r * (K + 1) + K] * eca, o = foa[r * K] * eoa[0].y;
    e = fmadd(feb[r * (K + 1) + K], ecb, e);
    e = fmadd(fea[r * (K + 1)], eoa[0].x, e);
    e = fmadd(feb[r * (K + 1)], eob[0].x, e);
    o = fmadd(fob[r * K], eob[0].y, o);
#pragma unroll
    for (int j = 1; j < K; ++j) {
      e = fmadd(fea[r * (K + 1) + j], eoa[j].x, e);
      o = fmadd(foa[r * K + j], eoa[j].y, o);
      e = fmadd(feb[r * (K + 1) + j], eob[j].x, e);
      o = fmadd(fob[r * K + j], eob[j].y, o);
    }
    out[r] = add_rn(e, o);
    out[M - 1 - r] = sub_rn(e, o);
  }
  T sc = fea[(K - 1) * (K + 1) + K] * eca;
  sc = fmadd(feb[(K - 1) * (K + 1) + K], ecb, sc);
#pragma unroll
  for (int j = 0; j < K; ++j) {
    sc = fmadd(fea[(K - 1) * (K + 1) + j], eoa[j].x, sc);
    sc = fmadd(feb[(K - 1) * (K + 1) + j], eob[j].x, sc);
  }
  out[K - 1] = sc;
}

// A u + B v with packed (even, odd) accumulators
template <int K, typename T>
__device__ __forceinline__ void fold_rows_sum2(const typename Pair<T>::type *fpa, const T *fea,
                                               const typename Pair<T>::type (&eoa)[K > 1 ? K : 1], const T eca,
                                               const typename Pair<T>::type *fpb, const T *feb,
                                               const typename Pair<T>::type (&eob)[K > 1 ? K : 1], const T ecb,
                                               T (&out)[2 * K - 1])
{
  using P = Pair<T>;
  constexpr int M = 2 * K - 1;
#pragma unroll
  for (int r = 0; r < K - 1; ++r) {
    typename P::type acc = P::make(fea[r * (K + 1) + K] * eca + feb[r * (K + 1) + K] * ecb, T(0));
#pragma unroll
    for (int j = 0; j < K; ++j) {
      acc = P::fma(fpa[r * K + j], eoa[j], acc);
      acc = P::fma(fpb[r * K + j], eob[j], acc);
    }
    out[r] = acc.x + acc.y;
    out[M - 1 - r] = acc.x - acc.y;
  }
  T sc = fea[(K - 1) * (K + 1) + K] * eca;
  sc += feb[(K - 1) * (K + 1) + K] * ecb;
#pragma unroll
  for (int j = 0; j < K; ++j) {
    sc += fea[(K - 1) * (K + 1) + j] * eoa[j].x;
    sc += feb[(K - 1) * (K + 1) + j] * eob[j].x;
  }
  out[K - 1] = sc;
}

// Fast-diagonalization factor S (eigenvectors as columns; modes 0..k-1 even,
// k..2k-2 odd) or its transpose applied to a line of 2k-1 values, with packed
// (even, odd) pairs.
template <int K, typename T, bool TRANSPOSE>
__device__ __forceinline__ void apply_evec2(const T (&in)[2 * K - 1], T (&out)[2 * K - 1])
{
  using P = Pair<T>;
  constexpr int M = 2 * K - 1, C = K - 1;
  const DegreeTables<K, T> &tb = c_tables<K, T>;
  if constexpr (TRANSPOSE) {
    typename P::type eo[C > 0 ? C : 1];
#pragma unroll
    for (int j = 0; j < C; ++j) eo[j] = P::make(in[j] + in[M - 1 - j], in[j] - in[M - 1 - j]);
    const T ec = in[C];
#pragma unroll
    for (int q = 0; q < C; ++q) {
      typename P::type acc = P::make(tb.evec[C * M + q] * ec, T(0));
#pragma unroll
      for (int j = 0; j < C; ++j) acc = P::fma(tb.evec_p[j * C + q], eo[j], acc);
      out[q] = acc.x;          // even mode q
      out[C + 1 + q] = acc.y;  // odd mode k+q
    }
    T sc = tb.evec[C * M + C] * ec;
#pragma unroll
    for (int j = 0; j < C; ++j) sc += tb.evec[j * M + C] * eo[j].x;
    out[C] = sc;
  } else {
#pragma unroll
    for (int i = 0; i < C; ++i) {
      typename P::type acc = P::make(tb.evec[i * M + C] * in[C], T(0));
#pragma unroll
      for (int q = 0; q < C; ++q) acc = P::fma(tb.evec_p[i * C + q], P::make(in[q], in[C + 1 + q]), acc);
      out[i] = acc.x + acc.y;
      out[M - 1 - i] = acc.x - acc.y;
    }
    T sc = T(0);
#pragma unroll
    for (int q = 0; q <= C; ++q) sc += tb.evec[C * M + q] * in[q];
    out[C] = sc;
  }
}

// patches per batch of autotuner variant v: 0 the default P, 1 P/2, 2 P/4
// (at least one patch; larger batches than P measured slower everywhere)
template <int K, typename T, int V>
constexpr int sm3_variant_ppb()
{
  constexpr int P = sm3_default_ppb<K, T>();
  if constexpr (V == 1) return P > 1 ? P / 2 : P;
  else if constexpr (V == 2) return P > 3 ? P / 4 : P;
  else return P;
}

// S or S^T with scalar FMAs (constant-bank coefficients); chains as in
// fold_rows_s: a product, then explicit fused multiply-adds in a fixed order;
// the even/odd combinations are unfusable adds (a chain of one product, at
// degree 2, would otherwise be fused into them)
template <int K, typename T, bool TRANSPOSE>
__device__ __forceinline__ void apply_evec_s(const T (&in)[2 * K - 1], T (&out)[2 * K - 1])
{
  constexpr int M = 2 * K - 1, C = K - 1;
  const DegreeTables<K, T> &tb = c_tables<K, T>;
  if constexpr (TRANSPOSE) {
    T ev[C > 0 ? C : 1], od[C > 0 ? C : 1];
#pragma unroll
    for (int j = 0; j < C; ++j) {
      ev[j] = in[j] + in[M - 1 - j];
      od[j] = in[j] - in[M - 1 - j];
    }
    const T ec = in[C];
#pragma unroll
    for (int q = 0; q < C; ++q) {
      T e = tb.evec[C * M + q] * ec, o = tb.evec[C + 1 + q] * od[0];
      e = fmadd(tb.evec[q], ev[0], e);
#pragma unroll
      for (int j = 1; j < C; ++j) {
        e = fmadd(tb.evec[j * M + q], ev[j], e);
        o = fmadd(tb.evec[j * M + C + 1 + q], od[j], o);
      }
      out[q] = e;
      out[C + 1 + q] = o;
    }
    T sc = tb.evec[C * M + C] * ec;
#pragma unroll
    for (int j = 0; j < C; ++j) sc = fmadd(tb.evec[j * M + C], ev[j], sc);
    out[C] = sc;
  } else {
#pragma unroll
    for (int i = 0; i < C; ++i) {
      T e = tb.evec[i * M + C] * in[C], o = tb.evec[i * M + C + 1] * in[C + 1];
      e = fmadd(tb.evec[i * M], in[0], e);
#pragma unroll
      for (int q = 1; q < C; ++q) {
        e = fmadd(tb.evec[i * M + q], in[q], e);
        o = fmadd(tb.evec[i * M + C + 1 + q], in[C + 1 + q], o);
      }
      out[i] = add_rn(e, o);
      out[M - 1 - i] = sub_rn(e, o);
    }
    T sc = tb.evec[C * M] * in[0];
#pragma unroll
    for (int q = 1; q <= C; ++q) sc = fmadd(tb.evec[C * M + q], in[q], sc);
    out[C] = sc;
  }
}

#ifndef TPS_SM3_PACKED
#define TPS_SM3_PACKED 0
#endif
#ifndef TPS_SM3_PACKED_MIN_K
#define TPS_SM3_PACKED_MIN_K 6
#endif
// packed (even, odd) pair contractions from degree 6 up, scalar below.
// Measured on B200, ms per 32^3 sweep, CTA kernel, scalar vs packed: Q7 FP32
// 0.820 vs 0.679, FP64 1.668 vs 1.620; Q6 FP32 0.500 vs 0.476, FP64 1.115 vs
// 1.035; at Q4 the two were within 1.5 %.  (Two-product sums as separate
// products and an add instead of one chain measured slower at every degree.)
template <int K>
constexpr bool sm3_packed()
{
  return TPS_SM3_PACKED != 0 || K >= TPS_SM3_PACKED_MIN_K;
}
template <int K, typename T>
__device__ __forceinline__ void rows_mass(const typename Pair<T>::type (&eo)[K > 1 ? K : 1], const T ec,
                                          T (&out)[2 * K - 1])
{
  const DegreeTables<K, T> &tb = c_tables<K, T>;
  if constexpr (sm3_packed<K>()) fold_rows2<K, T>(tb.pmass_fp, tb.pmass_fe, eo, ec, out);
  else fold_rows_s<K, T>(tb.pmass_fe, tb.pmass_fo, eo, ec, out);
}
template <int K, typename T>
__device__ __forceinline__ void rows_lap(const typename Pair<T>::type (&eo)[K > 1 ? K : 1], const T ec,
                                         T (&out)[2 * K - 1])
{
  const DegreeTables<K, T> &tb = c_tables<K, T>;
  if constexpr (sm3_packed<K>()) fold_rows2<K, T>(tb.plap_fp, tb.plap_fe, eo, ec, out);
  else fold_rows_s<K, T>(tb.plap_fe, tb.plap_fo, eo, ec, out);
}
// interior rows of M u + L v (patch mass and stiffness)
template <int K, typename T>
__device__ __forceinline__ void rows_mass_lap(const typename Pair<T>::type (&eou)[K > 1 ? K : 1], const T ecu,
                                              const typename Pair<T>::type (&eov)[K > 1 ? K : 1], const T ecv,
                                              T (&out)[2 * K - 1])
{
  const DegreeTables<K, T> &tb = c_tables<K, T>;
  if constexpr (sm3_packed<K>())
    fold_rows_sum2<K, T>(tb.pmass_fp, tb.pmass_fe, eou, ecu, tb.plap_fp, tb.plap_fe, eov, ecv, out);
  else
    fold_rows_sum_s<K, T>(tb.pmass_fe, tb.pmass_fo, eou, ecu, tb.plap_fe, tb.plap_fo, eov, ecv, out);
}
template <int K, typename T, bool TRANSPOSE>
__device__ __forceinline__ void evec_apply(const T (&in)[2 * K - 1], T (&out)[2 * K - 1])
{
  if constexpr (sm3_packed<K>()) apply_evec2<K, T, TRANSPOSE>(in, out);
  else apply_evec_s<K, T, TRANSPOSE>(in, out);
}

struct Sm3Args {
  int nx_c, ny_c, n_patches;  // patch lattice of the colour
  int cx, cy, cz;             // colour parities
  int n_batches;
  int zero_x;                 // x == 0 on entry (first colour of a zero-initialised sweep)
  int64_t sy, sz;             // vector pitches (elements)
  // n / nx_c == (n * mx) >> sx and n / (nx_c ny_c) == (n * mxy) >> sxy for
  // 0 <= n < 2^31 (see magic_div)
  uint32_t mx, sx, mxy, sxy;
};



template <int K, typename T, bool USE_TMA, int PPB_ = 0>
__global__ void __launch_bounds__(Sm3<K, T, PPB_>::NT)
    smoother3d_kernel(const __grid_constant__ CUtensorMap map_x,
                      const __grid_constant__ CUtensorMap map_b, T *__restrict__ x,
                      const T *__restrict__ b, const Sm3Args a, T scale, T fd_scale,
                      int *__restrict__ err)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  using S = Sm3<K, T, PPB_>;
  using P2 = typename Pair<T>::type;
  constexpr int N1 = S::N1, M = S::M, W = S::W, PPB = S::PPB, NT = S::NT, AL = S::A;
  const DegreeTables<K, T> &tb = c_tables<K, T>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T *sm = reinterpret_cast<T *>(smem_raw);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + S::TAIL_BAR);
  int &s_ok = *reinterpret_cast<int *>(smem_raw + S::TAIL_BAR + 16);
  int64_t *s_base = reinterpret_cast<int64_t *>(smem_raw + S::TAIL_BASE);
  int *s_xo = reinterpret_cast<int *>(smem_raw + S::TAIL_XO);
  const int tid = threadIdx.x;

  // patch j of the colour -> first DoF coordinates of its box
  auto patch_xyz = [&](int j, int &fx, int &fy, int &fz) {
    const int jz = fast_div(j, a.mxy, a.sxy), rz = j - jz * (a.nx_c * a.ny_c);
    const int jy = fast_div(rz, a.mx, a.sx), jx = rz - jy * a.nx_c;
    fx = (a.cx + 2 * jx) * K;
    fy = (a.cy + 2 * jy) * K;
    fz = (a.cz + 2 * jz) * K;
  };

  // fd_scale / (lambda_x + lambda_y + lambda_z) for every mode triple
  T *RL = sm + S::OFF_RL;
  for (int e = tid; e < S::QSZ; e += NT)
    RL[e] = fd_scale / (tb.eval[e % M] + tb.eval[(e / M) % M] + tb.eval[e / (M * M)]);
  if constexpr (USE_TMA) {
    if (tid == 0) {
      mbar_init(&bars[0], 1);
      mbar_init(&bars[1], 1);
      fence_mbar_init();
    }
  }
  __syncthreads();

  // issue the TMA loads of batch `bt` into stage `st` (one thread)
  auto issue = [&](int bt, int st) {
    T *stage = sm + st * PPB * S::STAGE;
    const int np = min(PPB, a.n_patches - bt * PPB);
    const uint32_t bytes = np * sizeof(T) * (S::BBOX + (a.zero_x ? 0 : S::XBOX));
    mbar_arrive_expect_tx(&bars[st], bytes);
    for (int lp = 0; lp < np; ++lp) {
      int fx, fy, fz;
      patch_xyz(bt * PPB + lp, fx, fy, fz);
      const int x0 = fx & ~(AL - 1);
      T *dst = stage + lp * S::STAGE;
      if (!a.zero_x) tma_load_3d(dst, &map_x, &bars[st], x0, fy, fz);
      tma_load_3d(dst + S::BOFF, &map_b, &bars[st], x0, fy + 1, fz + 1);
    }
  };

  if constexpr (USE_TMA) {
    if (tid == 0 && blockIdx.x < a.n_batches) issue(blockIdx.x, 0);
  }

  int it = 0;
  for (int bt = blockIdx.x; bt < a.n_batches; bt += gridDim.x, ++it) {
    const int st = USE_TMA ? (it & 1) : 0;
    T *stage = sm + st * PPB * S::STAGE;
    const int np = min(PPB, a.n_patches - bt * PPB);
    // per-batch patch offsets (threads 1..PPB while thread 0 waits for TMA)
    if (tid >= 1 && tid <= PPB) {
      const int lp = tid - 1;
      int fx, fy, fz;
      patch_xyz(bt * PPB + (lp < np ? lp : 0), fx, fy, fz);
      s_base[lp] = lp < np ? fx + 1 + (fy + 1) * a.sy + (fz + 1) * a.sz : int64_t(-1);
      s_xo[lp] = USE_TMA ? (fx & (AL - 1)) : 0;
    }
    if constexpr (USE_TMA) {
      if (tid == 0) {
        const int nb = bt + gridDim.x;
        if (nb < a.n_batches) {
          fence_proxy_async_smem();
          issue(nb, st ^ 1);
        }
        s_ok = mbar_wait_bounded(&bars[st], (it >> 1) & 1) ? 1 : 0;
        if (!s_ok) atomicExch(err, 1);
      }
      __syncthreads();
      if (!s_ok) return;  // uniform: every thread read the same flag
    } else {
      // plain coalesced loads (any pitch); the box is staged at x offset 0.
      // Chunks of independent loads are issued before their shared stores.
      constexpr int NX = PPB * N1 * N1 * N1, NB = PPB * M * M * M;
      constexpr int LX = (NX + NT - 1) / NT, LB = (NB + NT - 1) / NT, CH = 8;
#pragma unroll 1
      for (int i0 = 0; i0 < LX; i0 += CH) {
        T v[CH];
#pragma unroll
        for (int c = 0; c < CH; ++c) {
          const int e = tid + (i0 + c) * NT;
          const int lp = e / (N1 * N1 * N1), l = e % (N1 * N1 * N1);
          const int lx = l % N1, ly = (l / N1) % N1, lz = l / (N1 * N1);
          v[c] = T(0);
          if (i0 + c < LX && e < NX && lp < np && !a.zero_x) {
            int fx, fy, fz;
            patch_xyz(bt * PPB + lp, fx, fy, fz);
            v[c] = x[(fx + lx) + (fy + ly) * a.sy + (fz + lz) * a.sz];
          }
        }
#pragma unroll
        for (int c = 0; c < CH; ++c) {
          const int e = tid + (i0 + c) * NT;
          if (i0 + c < LX && e < NX) {
            const int lp = e / (N1 * N1 * N1), l = e % (N1 * N1 * N1);
            const int lx = l % N1, ly = (l / N1) % N1, lz = l / (N1 * N1);
            stage[lp * S::STAGE + (lz * N1 + ly) * W + lx] = v[c];
          }
        }
      }
#pragma unroll 1
      for (int i0 = 0; i0 < LB; i0 += CH) {
        T v[CH];
#pragma unroll
        for (int c = 0; c < CH; ++c) {
          const int e = tid + (i0 + c) * NT;
          const int lp = e / (M * M * M), l = e % (M * M * M);
          const int lx = l % M, ly = (l / M) % M, lz = l / (M * M);
          v[c] = T(0);
          if (i0 + c < LB && e < NB && lp < np) {
            int fx, fy, fz;
            patch_xyz(bt * PPB + lp, fx, fy, fz);
            v[c] = __ldg(&b[(fx + lx + 1) + (fy + ly + 1) * a.sy + (fz + lz + 1) * a.sz]);
          }
        }
#pragma unroll
        for (int c = 0; c < CH; ++c) {
          const int e = tid + (i0 + c) * NT;
          if (i0 + c < LB && e < NB) {
            const int lp = e / (M * M * M), l = e % (M * M * M);
            const int lx = l % M, ly = (l / M) % M, lz = l / (M * M);
            stage[lp * S::STAGE + S::BOFF + (lz * M + ly) * W + lx + 1] = v[c];
          }
        }
      }
      __syncthreads();
    }

    T *Z1 = sm + S::OFF_Z1, *Z2 = sm + S::OFF_Z2;
    // V1/V2 of patch lp at stage + lp*STAGE (+VSZ): the x box is dead after the z stage
    T *V1 = stage, *V2 = stage + S::VSZ;
    constexpr int VST = S::STAGE;  // V1/V2 patch stride
    T *Q1 = Z1, *Q2 = Z2;          // the fast-diagonalization stages reuse the Z arrays

    if (!a.zero_x) {
      // ---- z: Z1 = M_z x~, Z2 = L_z x~ (x~ = x with zero interior) ----------
      // ring lines (y or x on the box boundary) first, then pairs of interior lines
      for (int t = tid; t < PPB * (S::RING + S::IPAIR); t += NT) {
        if (t < PPB * S::RING) {
          const int lp = t / S::RING, r = t % S::RING;
          int y, xx;
          if (r < N1) {
            y = 0;
            xx = r;
          } else if (r < 2 * N1) {
            y = N1 - 1;
            xx = r - N1;
          } else {
            const int q = r - 2 * N1;
            y = 1 + (q >> 1);
            xx = (q & 1) ? N1 - 1 : 0;
          }
          const T *src = stage + lp * S::STAGE + y * W + s_xo[lp] + xx;
          T v[N1], ec, r1[M], r2[M];
          P2 eo[K > 1 ? K : 1];
#pragma unroll
          for (int z = 0; z < N1; ++z) v[z] = src[z * N1 * W];
          fold_pairs<K, T>(v, eo, ec);
          rows_mass<K, T>(eo, ec, r1);
          rows_lap<K, T>(eo, ec, r2);
          T *d1 = Z1 + lp * S::ZSZ + y * N1 + xx, *d2 = Z2 + lp * S::ZSZ + y * N1 + xx;
#pragma unroll
          for (int i = 0; i < M; ++i) {
            d1[i * N1 * N1] = r1[i];
            d2[i * N1 * N1] = r2[i];
          }
        } else {
          const int u = t - PPB * S::RING;
          const int lp = u / S::IPAIR, r0 = 2 * (u % S::IPAIR);
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int r = r0 + h;
            if (r >= M * M) break;
            const int y = 1 + r / M, xx = 1 + r % M;
            const T *src = stage + lp * S::STAGE + y * W + s_xo[lp] + xx;
            const T v0 = src[0], vn = src[(N1 - 1) * N1 * W];
            T *d1 = Z1 + lp * S::ZSZ + y * N1 + xx, *d2 = Z2 + lp * S::ZSZ + y * N1 + xx;
#pragma unroll
            for (int i = 0; i < M; ++i) {
              d1[i * N1 * N1] = fmadd(tb.pmass[(i + 1) * N1 + N1 - 1], vn, tb.pmass[(i + 1) * N1] * v0);
              d2[i * N1 * N1] = fmadd(tb.plap[(i + 1) * N1 + N1 - 1], vn, tb.plap[(i + 1) * N1] * v0);
            }
          }
        }
      }
      __syncthreads();
      // ---- y: V1 = M_y Z2 + L_y Z1, V2 = M_y Z1 ------------------------------
      for (int t = tid; t < PPB * M * N1; t += NT) {
        const int lp = t / (M * N1), r = t % (M * N1);
        const int zi = r / N1, xx = r % N1;
        const T *s1 = Z1 + lp * S::ZSZ + zi * N1 * N1 + xx;
        const T *s2 = Z2 + lp * S::ZSZ + zi * N1 * N1 + xx;
        T v[N1], ec1, ec2;
        P2 eo1[K > 1 ? K : 1], eo2[K > 1 ? K : 1];
#pragma unroll
        for (int j = 0; j < N1; ++j) v[j] = s1[j * N1];
        fold_pairs<K, T>(v, eo1, ec1);
#pragma unroll
        for (int j = 0; j < N1; ++j) v[j] = s2[j * N1];
        fold_pairs<K, T>(v, eo2, ec2);
        T ra[M], rc[M];
        rows_mass_lap<K, T>(eo2, ec2, eo1, ec1, ra);
        rows_mass<K, T>(eo1, ec1, rc);
        T *d1 = V1 + lp * VST + zi * M * N1 + xx, *d2 = V2 + lp * VST + zi * M * N1 + xx;
#pragma unroll
        for (int i = 0; i < M; ++i) {
          d1[i * N1] = ra[i];
          d2[i * N1] = rc[i];
        }
      }
      __syncthreads();
    }
    // ---- x: r = b - s (M_x V1 + L_x V2), then S^T along x -> Q1 -----------
    for (int t = tid; t < PPB * M * M; t += NT) {
      const int lp = t / (M * M), r = t % (M * M);  // r = zi * M + yi
      T res[M];
      const T *bb = stage + lp * S::STAGE + S::BOFF + r * W + s_xo[lp] + 1;
      if (!a.zero_x) {
        const T *s1 = V1 + lp * VST + r * N1, *s2 = V2 + lp * VST + r * N1;
        T v[N1], ec1, ec2;
        P2 eo1[K > 1 ? K : 1], eo2[K > 1 ? K : 1];
#pragma unroll
        for (int j = 0; j < N1; ++j) v[j] = s1[j];
        fold_pairs<K, T>(v, eo1, ec1);
#pragma unroll
        for (int j = 0; j < N1; ++j) v[j] = s2[j];
        fold_pairs<K, T>(v, eo2, ec2);
        T ra[M];
        rows_mass_lap<K, T>(eo1, ec1, eo2, ec2, ra);
#pragma unroll
        for (int i = 0; i < M; ++i) res[i] = bb[i] - scale * ra[i];
      } else {
#pragma unroll
        for (int i = 0; i < M; ++i) res[i] = bb[i];
      }
      T q[M];
      evec_apply<K, T, true>(res, q);
      T *d = Q1 + lp * S::QSZ + r * M;
#pragma unroll
      for (int i = 0; i < M; ++i) d[i] = q[i];
    }
    __syncthreads();
    // ---- S^T along y: Q1 -> Q2 -------------------------------------------
    for (int t = tid; t < PPB * M * M; t += NT) {
      const int lp = t / (M * M), r = t % (M * M);
      const int zi = r / M, qx = r % M;
      const T *s = Q1 + lp * S::QSZ + zi * M * M + qx;
      T v[M], q[M];
#pragma unroll
      for (int j = 0; j < M; ++j) v[j] = s[j * M];
      evec_apply<K, T, true>(v, q);
      T *d = Q2 + lp * S::QSZ + zi * M * M + qx;
#pragma unroll
      for (int j = 0; j < M; ++j) d[j * M] = q[j];
    }
    __syncthreads();
    // ---- S^T along z, eigenvalue scaling, S along z: Q2 -> Q1 ---------------
    for (int t = tid; t < PPB * M * M; t += NT) {
      const int lp = t / (M * M), r = t % (M * M);
      const T *s = Q2 + lp * S::QSZ + r;
      T v[M], q[M];
#pragma unroll
      for (int j = 0; j < M; ++j) v[j] = s[j * M * M];
      evec_apply<K, T, true>(v, q);
#pragma unroll
      for (int j = 0; j < M; ++j) q[j] *= RL[j * M * M + r];
      evec_apply<K, T, false>(q, v);
      T *d = Q1 + lp * S::QSZ + r;
#pragma unroll
      for (int j = 0; j < M; ++j) d[j * M * M] = v[j];
    }
    __syncthreads();
    // ---- S along x: Q1 -> Q2 ---------------------------------------------
    for (int t = tid; t < PPB * M * M; t += NT) {
      const int lp = t / (M * M), r = t % (M * M);
      const T *s = Q1 + lp * S::QSZ + r * M;
      T v[M], q[M];
#pragma unroll
      for (int j = 0; j < M; ++j) v[j] = s[j];
      evec_apply<K, T, false>(v, q);
      T *d = Q2 + lp * S::QSZ + r * M;
#pragma unroll
      for (int j = 0; j < M; ++j) d[j] = q[j];
    }
    __syncthreads();
    // ---- S along y and store x_I -----------------------------------------
    for (int t = tid; t < PPB * M * M; t += NT) {
      const int lp = t / (M * M), r = t % (M * M);
      const int z = r / M, xx = r % M;
      const T *s = Q2 + lp * S::QSZ + z * M * M + xx;
      T v[M], q[M];
#pragma unroll
      for (int j = 0; j < M; ++j) v[j] = s[j * M];
      evec_apply<K, T, false>(v, q);
      const int64_t base = s_base[lp];
      if (base >= 0) {
        T *dst = x + base + xx + z * a.sz;
#pragma unroll
        for (int j = 0; j < M; ++j) dst[j * a.sy] = q[j];
      }
    }
    __syncthreads();  // every read of this stage is done before it is refilled
  }
}

}  // namespace tps
