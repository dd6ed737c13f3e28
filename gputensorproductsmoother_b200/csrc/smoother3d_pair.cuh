// 3D fused vertex-patch smoother, FP32, two patches per warp in packed
// FP32x2 arithmetic (sm_100a).
//
// Same per-patch algebra, contraction order and rounding as
// smoother3d_warp_kernel and smoother3d_kernel (the reference's FUSED_CF
// patch kernel, include/loop_kernel.cuh:962-1060 with
// include/evaluate_kernel.cuh:501-590, 1327-1434, 2058-2163): box residual
// b - A x~ with the interior of x set to zero, then the fast-diagonalisation
// solve and the store of omega A_II^{-1} r_I.  Every value of the staged
// intermediates is a pair (patch A, patch B), every multiply-add is one
// fma.rn.f32x2 over the pair with the coefficient in both halves, so each
// patch sees exactly the scalar kernels' operations: the sweeps are
// bit-identical (up to the sign of zero results).
//
// Why pairs: the one-warp-per-patch kernel is bound by instruction issue
// (about 1,700 warp instructions per Q4 patch, the shared-memory pipe 68 %
// busy).  Here one instruction serves two patches for the arithmetic, the
// shared-memory traffic of the intermediates (64-bit accesses), the address
// arithmetic and the loop/TMA skeleton; only the raw box and b-slab reads
// and the global stores stay per patch.
//
// Execution model: a team of warps -- one CTA, two warps from degree 4 on --
// owns its pairs of patches (patches 2q and 2q+1 of the colour, q = pair
// index), one stage and one mbarrier.  Every stage's work is a list of 32-lane
// passes; warp w of the team takes passes w, w + TEAM, ..., so a pair moves
// through its stages with the team's warps side by side and twice the warps
// per SM share the same shared memory (the kernel is latency-bound: more
// resident warps, not fewer instructions, is what it lacks).  Stages are
// separated by the team's barrier; the next pair's two x boxes and two b
// slabs are fetched by TMA (4 copies on one mbarrier) as soon as the x stage
// has consumed the current ones.  An odd last patch is paired with itself
// and stored once.  Every wait is bounded.
//
// Shared memory (8-byte pair elements): the z-stage outputs are kept only
// for the 8k ring lines of the box face.  On the interior lines x~ is zero
// except on the two z faces, so the z stage stores just those two values
// and the y stage forms the z products itself, with the same rounding.  That
// is 4.7 KB less per team at degree 4 (Q3 64^3 sweep 0.253 -> 0.228 ms).
// The z- and y-stage outputs are stored task-major for the stage that reads
// them (consecutive or shared words); the four fast-diagonalisation arrays
// use the 8-byte layouts WpLayout<K, 8>.  Every
// stage runs its passes as straight-line code: lanes past the last task redo
// a valid task and skip the stores, so the loads of one pass can be issued
// while the previous pass computes (lanes past the last task take task
// lane mod the task count, which is a valid task at every degree).
#pragma once

#include <cuda.h>

#include "ptx.cuh"
#include "smoother3d.cuh"
#include "smoother3d_warp.cuh"
#include "tps_common.cuh"

namespace tps {

// ---- packed pair arithmetic (patch A in .x, patch B in .y) -------------------
__device__ __forceinline__ float2 pr_bc(float c) { return make_float2(c, c); }
__device__ __forceinline__ float2 pr_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 pr_sub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 pr_mul(float c, float2 a) { return __fmul2_rn(pr_bc(c), a); }
__device__ __forceinline__ float2 pr_fma(float c, float2 a, float2 acc) { return __ffma2_rn(pr_bc(c), a, acc); }

// v (2k+1 pairs) -> even sums E_j, odd differences O_j (j < k), centre ec
template <int K>
__device__ __forceinline__ void pr_fold(const float2 (&v)[2 * K + 1], float2 (&E)[K], float2 (&O)[K], float2 &ec)
{
#pragma unroll
  for (int j = 0; j < K; ++j) {
    E[j] = pr_add(v[j], v[2 * K - j]);
    O[j] = pr_sub(v[j], v[2 * K - j]);
  }
  ec = v[K];
}

// interior rows of one centro-symmetric patch matrix (fold_rows_s, the same
// chains and order)
template <int K>
__device__ __forceinline__ void pr_rows(const float *fe, const float *fo, const float2 (&E)[K], const float2 (&O)[K],
                                        const float2 ec, float2 (&out)[2 * K - 1])
{
  constexpr int M = 2 * K - 1;
#pragma unroll
  for (int r = 0; r < K - 1; ++r) {
    float2 e = pr_mul(fe[r * (K + 1) + K], ec), o = pr_mul(fo[r * K], O[0]);
    e = pr_fma(fe[r * (K + 1)], E[0], e);
#pragma unroll
    for (int j = 1; j < K; ++j) {
      e = pr_fma(fe[r * (K + 1) + j], E[j], e);
      o = pr_fma(fo[r * K + j], O[j], o);
    }
    out[r] = pr_add(e, o);
    out[M - 1 - r] = pr_sub(e, o);
  }
  float2 sc = pr_mul(fe[(K - 1) * (K + 1) + K], ec);
#pragma unroll
  for (int j = 0; j < K; ++j) sc = pr_fma(fe[(K - 1) * (K + 1) + j], E[j], sc);
  out[K - 1] = sc;
}

// interior rows of A u + B v with one accumulation chain (fold_rows_sum_s)
template <int K>
__device__ __forceinline__ void pr_rows_sum(const float *fea, const float *foa, const float2 (&Ea)[K],
                                            const float2 (&Oa)[K], const float2 eca, const float *feb,
                                            const float *fob, const float2 (&Eb)[K], const float2 (&Ob)[K],
                                            const float2 ecb, float2 (&out)[2 * K - 1])
{
  constexpr int M = 2 * K - 1;
#pragma unroll
  for (int r = 0; r < K - 1; ++r) {
    float2 e = pr_mul(fea[r * (K + 1) + K], eca), o = pr_mul(foa[r * K], Oa[0]);
    e = pr_fma(feb[r * (K + 1) + K], ecb, e);
    e = pr_fma(fea[r * (K + 1)], Ea[0], e);
    e = pr_fma(feb[r * (K + 1)], Eb[0], e);
    o = pr_fma(fob[r * K], Ob[0], o);
#pragma unroll
    for (int j = 1; j < K; ++j) {
      e = pr_fma(fea[r * (K + 1) + j], Ea[j], e);
      o = pr_fma(foa[r * K + j], Oa[j], o);
      e = pr_fma(feb[r * (K + 1) + j], Eb[j], e);
      o = pr_fma(fob[r * K + j], Ob[j], o);
    }
    out[r] = pr_add(e, o);
    out[M - 1 - r] = pr_sub(e, o);
  }
  float2 sc = pr_mul(fea[(K - 1) * (K + 1) + K], eca);
  sc = pr_fma(feb[(K - 1) * (K + 1) + K], ecb, sc);
#pragma unroll
  for (int j = 0; j < K; ++j) {
    sc = pr_fma(fea[(K - 1) * (K + 1) + j], Ea[j], sc);
    sc = pr_fma(feb[(K - 1) * (K + 1) + j], Eb[j], sc);
  }
  out[K - 1] = sc;
}

// S or S^T on a line of 2k-1 pairs (apply_evec_s, the same chains and order)
template <int K, bool TRANSPOSE>
__device__ __forceinline__ void pr_evec(const float2 (&in)[2 * K - 1], float2 (&out)[2 * K - 1])
{
  constexpr int M = 2 * K - 1, C = K - 1;
  const DegreeTables<K, float> &tb = c_tables<K, float>;
  if constexpr (TRANSPOSE) {
    float2 ev[C > 0 ? C : 1], od[C > 0 ? C : 1];
#pragma unroll
    for (int j = 0; j < C; ++j) {
      ev[j] = pr_add(in[j], in[M - 1 - j]);
      od[j] = pr_sub(in[j], in[M - 1 - j]);
    }
    const float2 ec = in[C];
#pragma unroll
    for (int q = 0; q < C; ++q) {
      float2 e = pr_mul(tb.evec[C * M + q], ec), o = pr_mul(tb.evec[C + 1 + q], od[0]);
      e = pr_fma(tb.evec[q], ev[0], e);
#pragma unroll
      for (int j = 1; j < C; ++j) {
        e = pr_fma(tb.evec[j * M + q], ev[j], e);
        o = pr_fma(tb.evec[j * M + C + 1 + q], od[j], o);
      }
      out[q] = e;
      out[C + 1 + q] = o;
    }
    float2 sc = pr_mul(tb.evec[C * M + C], ec);
#pragma unroll
    for (int j = 0; j < C; ++j) sc = pr_fma(tb.evec[j * M + C], ev[j], sc);
    out[C] = sc;
  } else {
#pragma unroll
    for (int i = 0; i < C; ++i) {
      float2 e = pr_mul(tb.evec[i * M + C], in[C]), o = pr_mul(tb.evec[i * M + C + 1], in[C + 1]);
      e = pr_fma(tb.evec[i * M], in[0], e);
#pragma unroll
      for (int q = 1; q < C; ++q) {
        e = pr_fma(tb.evec[i * M + q], in[q], e);
        o = pr_fma(tb.evec[i * M + C + 1 + q], in[C + 1 + q], o);
      }
      out[i] = pr_add(e, o);
      out[M - 1 - i] = pr_sub(e, o);
    }
    float2 sc = pr_mul(tb.evec[C * M], in[0]);
#pragma unroll
    for (int q = 1; q <= C; ++q) sc = pr_fma(tb.evec[C * M + q], in[q], sc);
    out[C] = sc;
  }
}

// degrees with a compiled pair kernel (FP32; the scalar folded contractions
// of degrees <= 5 are the ones it mirrors)
template <int K>
constexpr bool pp3_enabled()
{
  return K >= 2 && K <= 5;
}

template <int K, int TEAM>
struct Pp3 {
  using L = WpLayout<K, 8>;  // strides of the 8-byte pair elements
  static constexpr int N1 = 2 * K + 1, M = 2 * K - 1;
  static constexpr int A = Sm3<K, float>::A, W = Sm3<K, float>::W;  // TMA boxes as the FP32 kernels'
  static constexpr int XBOX = N1 * N1 * W, BBOX = M * M * W;        // floats per patch
  static constexpr int ALIGN = 32;                                   // floats (128 B: TMA destinations)
  static constexpr int XBOX_A = wp_rup(XBOX, ALIGN), BBOX_A = wp_rup(BBOX, ALIGN);
  // The z stage's output for the box face lines, in "task-major" layouts
  // (the reading stage's task is the fastest index, so its reads are
  // consecutive or shared words):
  // * ring lines (the RING = 8K lines with y or x on the box face), ring
  //   index q: top row q = x, bottom row N1 + x, left column 2 N1 + y - 1,
  //   right column 2 N1 + M + y - 1; ZR1 = M_z x~ and ZR2 = L_z x~ as
  //   [q][zi] (zi fastest);
  // * interior lines (y, x both interior): x~ is zero there except on the
  //   z faces, so M_z x~ = m_0 x(0) + m_N x(N1 - 1) per output; only the two
  //   face values are kept, F0 and F8 as [y - 1][x - 1], and the y stage
  //   forms the products itself, with the same rounding as the z stage's
  //   ring lines.
  // V [zi][yi][x] with strides VL (x stride M * M chosen by a bank-conflict
  // search over the y stage's lane mapping).
  static constexpr int RING = N1 * N1 - M * M, IPAIR = (M * M + 1) / 2;
  static constexpr int ZR = RING * M, ZI = M * M;  // pair elements of ZR1 / ZR2 and of F0 / F8
  // F0 starts PADF pair elements after ZR2: at degree 4 that puts the y
  // stage's reads of F0 and F8 (interior columns) on other bank pairs than
  // its reads of ZR1 and ZR2 (side columns) in the same instruction
  // (F0 and F8 at words 5 and 6 mod 16; by a wavefront model of both passes)
  static constexpr int PADF = K == 4 ? 5 : 0;
  static constexpr Str3 VL{M, 1, M * M};           // {zi, yi, x} strides of V
  static constexpr int VEXT = (M - 1) * VL.p + (M - 1) * VL.r + (N1 - 1) * VL.c + 1;
  static constexpr int NZP = (RING + IPAIR + 31) / 32;  // passes of the z stage
  static constexpr int ext(Str3 s) { return (M - 1) * (s.p + s.r + s.c) + 1; }
  static constexpr int QBUF1 = wp_max(ext(L::QA), ext(L::QC)), QBUF2 = wp_max(ext(L::QB), ext(L::QD));
  // per team (floats): [x box A | x box B, later V1 | V2] [b slab A | b slab B]
  // [ZR1 | ZR2 | F0 | F8, later QA/QC | QB/QD]; pair arrays take 2 floats per element
  static constexpr int BOFF = wp_rup(wp_max(2 * XBOX_A, 4 * VEXT), ALIGN);
  static constexpr int ZOFF = BOFF + 2 * BBOX_A;
  static constexpr int ZSPAN = wp_max(4 * (ZR + ZI) + 2 * PADF, 2 * (QBUF1 + QBUF2));
  static constexpr int WARP_ELEMS = wp_rup(ZOFF + ZSPAN, ALIGN);
  static constexpr int NT = 32 * TEAM;  // one team = one CTA, one pair of patches at a time
  // the eigenvalue scalings live in registers (no shared table), so that the
  // stage alone sets the CTAs per SM; the mbarrier sits right after the stage
  static constexpr size_t OFF_BAR = (sizeof(float) * static_cast<size_t>(ZOFF + ZSPAN) + 7) / 8 * 8;
  static constexpr size_t BYTES = OFF_BAR + 8;
  static constexpr int NZT = RING + IPAIR, NYT = M * N1, NQT = M * M;
  // 32-lane passes of each stage; warp w of the team takes passes w, w + TEAM, ...
  static constexpr int NYP = (NYT + 31) / 32, NP = (NQT + 31) / 32;
  static constexpr int NZPW = (NZP + TEAM - 1) / TEAM, NYPW = (NYP + TEAM - 1) / TEAM, NPW = (NP + TEAM - 1) / TEAM;
};

// z-stage task of a lane in one pass: ring = one full z-line (its ring
// index q is the task index t, so lane t's stores of ZR1 / ZR2 are the words
// t * M + zi: an odd stride, conflict-free), else up to two interior z-lines
// (interior indices i and i + IPAIR, consecutive across lanes); positions
// y * N1 + x, -1 = none
struct PairZTask {
  int ring, in0, in1;
};

template <int K>
__device__ __forceinline__ PairZTask pair_ztask(int lane, int p)
{
  constexpr int N1 = 2 * K + 1, M = 2 * K - 1, RING = N1 * N1 - M * M, IPAIR = (M * M + 1) / 2;
  constexpr int NZT = RING + IPAIR;
  PairZTask r{-1, -1, -1};
  const int t = lane + 32 * p;
  if (t < RING) {
    int y, xx;
    if (t < N1) {
      y = 0;
      xx = t;
    } else if (t < 2 * N1) {
      y = N1 - 1;
      xx = t - N1;
    } else if (t < 2 * N1 + M) {
      y = 1 + t - 2 * N1;
      xx = 0;
    } else {
      y = 1 + t - 2 * N1 - M;
      xx = N1 - 1;
    }
    r.ring = y * N1 + xx;
  } else if (t < NZT) {
    const int e0 = t - RING, e1 = e0 + IPAIR;
    r.in0 = (1 + e0 / M) * N1 + 1 + e0 % M;
    if (e1 < M * M) r.in1 = (1 + e1 / M) * N1 + 1 + e1 % M;
  }
  return r;
}

// Warps per pair of patches (the team, one CTA): two from degree 4 on, where
// every stage has at least two 32-lane passes, so the warps split a pair's
// passes and twice the warps per SM share the staged boxes' shared memory;
// one below.  The register bound (pp3_regs) follows from as many CTAs per
// SM as shared memory holds, but at most 16 warps' worth (a thread may then
// keep 128 registers), except at degree 4 (below).  The grid is sized by the
// occupancy the compiled kernel reaches.
constexpr int kPairMaxWarpsPerSm = 16;
template <int K>
constexpr int pp3_warps()
{
  return K >= 4 ? 2 : 1;
}
template <int K>
constexpr int pp3_ctas()
{
  constexpr int w = pp3_warps<K>();
  int ctas = static_cast<int>(233472 / (Pp3<K, w>::BYTES + 1024));  // 0: does not fit
  if (ctas * w > kPairMaxWarpsPerSm) ctas = kPairMaxWarpsPerSm / w;
  ctas = ctas > 32 ? 32 : ctas;
  return ctas < 1 ? 1 : ctas;
}

// registers a thread may keep: what pp3_ctas CTAs per SM leave, except at
// degree 4, where the bound is 88.  The kernel then uses 84 (ms per Q4 64^3
// sweep: 0.451, against 0.459 with 90).  Registers are allocated per SM
// sub-partition, 5 warps of 88 each, so 10 CTAs of two warps fit either way.
// A bound of 80 (6 warps per sub-partition, 11 CTAs with shared memory)
// measured 0.467.
template <int K>
constexpr int pp3_regs()
{
  if (K == 4) return 88;
  const int r = 65536 / (pp3_ctas<K>() * 32 * pp3_warps<K>()) / 8 * 8;
  return r > 255 ? 255 : r;
}

template <int K, int TEAM>
__global__ void __launch_bounds__(32 * TEAM) __maxnreg__(pp3_regs<K>())
    smoother3d_pair_kernel(const __grid_constant__ CUtensorMap map_x, const __grid_constant__ CUtensorMap map_b,
                           float *__restrict__ x, const Sm3Args a, float scale, float fd_scale,
                           int *__restrict__ err)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  using S = Pp3<K, TEAM>;
  using Lo = typename S::L;
  constexpr int N1 = S::N1, M = S::M, W = S::W, AL = S::A;
  constexpr Str3 QA = Lo::QA, QB = Lo::QB, QC = Lo::QC, QD = Lo::QD;
  const DegreeTables<K, float> &tb = c_tables<K, float>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int tid = threadIdx.x, lane = tid & 31, wt = tid >> 5;  // wt: warp within the team
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw + S::OFF_BAR);
  float *stage = reinterpret_cast<float *>(smem_raw);
  // the team's barrier between stages (one warp: the warp's own)
  auto team_sync = [&]() {
    if constexpr (TEAM == 1)
      __syncwarp();
    else
      __syncthreads();
  };
  float2 *ZR1 = reinterpret_cast<float2 *>(stage + S::ZOFF), *ZR2 = ZR1 + S::ZR;
  float2 *F0 = ZR2 + S::ZR + S::PADF, *F8 = F0 + S::ZI;
  float2 *V1 = reinterpret_cast<float2 *>(stage), *V2 = V1 + S::VEXT;
  float2 *QAb = ZR1, *QBb = ZR1 + S::QBUF1;  // QA and QC share one buffer, QB and QD the other
  const float *boxA = stage, *boxB = stage + S::XBOX_A;
  const float *bslA = stage + S::BOFF, *bslB = bslA + S::BBOX_A;

  if (tid == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  __syncthreads();  // the mbarrier is ready
  // this lane's eigenvalue scalings of the z stage of the solve (the tasks of
  // this warp's passes, modes 0..M-1), kept in registers: line t = (qy, qx) =
  // (t / M, t % M), mode qz = jj, omega / (s (lambda_qx + lambda_qy + lambda_qz))
  constexpr int NPW = S::NPW;
  float rl[NPW][M];
#pragma unroll
  for (int j = 0; j < NPW; ++j) {
    const int t0 = lane + 32 * (wt + TEAM * j);
    const int t = t0 < S::NQT ? t0 : lane % S::NQT;
    const float exy = tb.eval[t % M], eyy = tb.eval[t / M];
#pragma unroll
    for (int jj = 0; jj < M; ++jj) rl[j][jj] = fd_scale / (exy + eyy + tb.eval[jj]);
  }

  // this lane's y-stage lines (task t = (zi, xx) = (t % M, t / M), one per
  // pass of this warp): rows 1..M of a side column (xx = 0 or N1 - 1) are ring
  // lines, read from ZR1 / ZR2; those of an interior column are formed from
  // the face values F0 / F8 as c_0 x(0) + c_N x(N1 - 1) of row zi + 1 of the
  // patch mass and stiffness.  Side lanes take coefficients (1, 0) and (0, 1),
  // which pass the ring values through (up to the sign of a zero).
  float yc[S::NYPW][4];  // c_0 and c_N of the mass, then of the stiffness
  int yb[S::NYPW][2];    // offsets (pair elements from ZR1) of rows y = 1 of the two arrays
#pragma unroll
  for (int j = 0; j < S::NYPW; ++j) {
    const int t0 = lane + 32 * (wt + TEAM * j);
    const int t = t0 < S::NYT ? t0 : lane % S::NYT;
    const int zi = t % M, xx = t / M;
    const bool side = xx == 0 || xx == N1 - 1;
    yc[j][0] = side ? 1.f : tb.pmass[(zi + 1) * N1];
    yc[j][1] = side ? 0.f : tb.pmass[(zi + 1) * N1 + N1 - 1];
    yc[j][2] = side ? 0.f : tb.plap[(zi + 1) * N1];
    yc[j][3] = side ? 1.f : tb.plap[(zi + 1) * N1 + N1 - 1];
    yb[j][0] = side ? (2 * N1 + (xx == 0 ? 0 : M)) * M + zi : 2 * S::ZR + S::PADF + xx - 1;
    yb[j][1] = yb[j][0] + (side ? S::ZR : S::ZI);
  }

  const int n_pairs = (a.n_patches + 1) >> 1;
  const int G = gridDim.x;
  int q = blockIdx.x;
  // thread 0: both x boxes and b slabs of the pair with box origins (fA, fB)
  auto issue = [&](int fxa, int fya, int fza, int fxb, int fyb, int fzb) {
    mbar_arrive_expect_tx(bar, static_cast<uint32_t>(sizeof(float) * 2 * (S::BBOX + (a.zero_x ? 0 : S::XBOX))));
    if (!a.zero_x) {
      tma_load_3d(stage, &map_x, bar, fxa & ~(AL - 1), fya, fza);
      tma_load_3d(stage + S::XBOX_A, &map_x, bar, fxb & ~(AL - 1), fyb, fzb);
    }
    tma_load_3d(stage + S::BOFF, &map_b, bar, fxa & ~(AL - 1), fya + 1, fza + 1);
    tma_load_3d(stage + S::BOFF + S::BBOX_A, &map_b, bar, fxb & ~(AL - 1), fyb + 1, fzb + 1);
  };
  // pair q -> box origins of patches 2q and 2q+1 (the last patch twice for an odd count)
  auto pair_xyz = [&](int qq, int &fxa, int &fya, int &fza, int &fxb, int &fyb, int &fzb) {
    const int ja = 2 * qq, jb = ja + 1 < a.n_patches ? ja + 1 : ja;
    wp_patch_xyz(a, ja, K, fxa, fya, fza);
    wp_patch_xyz(a, jb, K, fxb, fyb, fzb);
  };
  PairZTask ztk[S::NZPW];  // this lane's z-stage lines, per pass of this warp
#pragma unroll
  for (int j = 0; j < S::NZPW; ++j) {
    const int p = wt + TEAM * j;
    ztk[j] = p < S::NZP ? pair_ztask<K>(lane, p) : PairZTask{-1, -1, -1};
  }
  int fxa = 0, fya = 0, fza = 0, fxb = 0, fyb = 0, fzb = 0;
  if (q < n_pairs) {
    pair_xyz(q, fxa, fya, fza, fxb, fyb, fzb);
    if (tid == 0) issue(fxa, fya, fza, fxb, fyb, fzb);
  }

  for (int it = 0; q < n_pairs; q += G, ++it) {
    const int xoa = fxa & (AL - 1), xob = fxb & (AL - 1);
    const bool store_b = 2 * q + 1 < a.n_patches;
    int nxa = 0, nya = 0, nza = 0, nxb = 0, nyb = 0, nzb = 0;  // the next pair of this team
    if (q + G < n_pairs) pair_xyz(q + G, nxa, nya, nza, nxb, nyb, nzb);
    const bool ok = mbar_wait_bounded(bar, it & 1);
    if (TEAM == 1 ? !__all_sync(0xffffffffu, ok) : !__syncthreads_and(ok)) {
      if (tid == 0) atomicExch(err, 1);
      return;  // the only copies in flight were the ones waited for
    }

    if (!a.zero_x) {
      // ---- z: ZR1 = M_z x~, ZR2 = L_z x~ on the ring lines; the face values
      // x(0), x(N1 - 1) of the interior lines into F0, F8 ----
      const float *ba = boxA + xoa, *bb = boxB + xob;
#pragma unroll
      for (int j = 0; j < S::NZPW; ++j) {
        const PairZTask tk = ztk[j];
        if (tk.ring >= 0) {
          const int q = lane + 32 * (wt + TEAM * j);  // ring index = task index
          const int y = tk.ring / N1, xx = tk.ring % N1;
          const int o = y * W + xx;
          float2 v[N1], E[K], O[K], ec, r1[M], r2[M];
#pragma unroll
          for (int z = 0; z < N1; ++z) v[z] = make_float2(ba[o + z * N1 * W], bb[o + z * N1 * W]);
          pr_fold<K>(v, E, O, ec);
          pr_rows<K>(tb.pmass_fe, tb.pmass_fo, E, O, ec, r1);
          pr_rows<K>(tb.plap_fe, tb.plap_fo, E, O, ec, r2);
          float2 *d1 = ZR1 + q * M, *d2 = ZR2 + q * M;
#pragma unroll
          for (int i = 0; i < M; ++i) {
            d1[i] = r1[i];
            d2[i] = r2[i];
          }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int pos = h == 0 ? tk.in0 : tk.in1;
          if (pos >= 0) {
            const int y = pos / N1, xx = pos % N1;
            const int o = y * W + xx, e = (y - 1) * M + xx - 1;
            F0[e] = make_float2(ba[o], bb[o]);
            F8[e] = make_float2(ba[o + (N1 - 1) * N1 * W], bb[o + (N1 - 1) * N1 * W]);
          }
        }
      }
      team_sync();
      // ---- y: V1 = M_y Z2 + L_y Z1, V2 = M_y Z1 (V overwrites the dead x boxes) ----
      // task t = (zi, xx) = (t % M, t / M); lanes past the last task redo a
      // valid task (lane mod the task count) and skip the stores, so every pass
      // is straight-line code.  Z1, Z2 on the lane's line: rows 0 and N1 - 1
      // from the ring arrays (ring index xx and N1 + xx, so word t and
      // N1 M + t), rows 1..M as set up above; folded in pairs of rows as
      // pr_fold does.
#pragma unroll
      for (int j = 0; j < S::NYPW; ++j) {
        const int t0 = lane + 32 * (wt + TEAM * j);
        const bool act = t0 < S::NYT;
        const int t = act ? t0 : lane % S::NYT;
        const int zi = t % M, xx = t / M;
        const float2 *s1 = ZR1 + yb[j][0], *s2 = ZR1 + yb[j][1];
        const float cm0 = yc[j][0], cmn = yc[j][1], cl0 = yc[j][2], cln = yc[j][3];
        // Z1, Z2 of row y = 1 + r of the line
        auto zrow = [&](int r, float2 &z1, float2 &z2) {
          const float2 f0 = s1[r * M], f8 = s2[r * M];
          z1 = pr_fma(cmn, f8, pr_mul(cm0, f0));
          z2 = pr_fma(cln, f8, pr_mul(cl0, f0));
        };
        float2 E1[K], O1[K], ec1, E2[K], O2[K], ec2;
        {
          const float2 a1 = ZR1[t], b1 = ZR1[N1 * M + t], a2 = ZR2[t], b2 = ZR2[N1 * M + t];
          E1[0] = pr_add(a1, b1);
          O1[0] = pr_sub(a1, b1);
          E2[0] = pr_add(a2, b2);
          O2[0] = pr_sub(a2, b2);
        }
#pragma unroll
        for (int jj = 1; jj < K; ++jj) {
          float2 a1, a2, b1, b2;
          zrow(jj - 1, a1, a2);          // row jj
          zrow(N1 - 2 - jj, b1, b2);     // row N1 - 1 - jj
          E1[jj] = pr_add(a1, b1);
          O1[jj] = pr_sub(a1, b1);
          E2[jj] = pr_add(a2, b2);
          O2[jj] = pr_sub(a2, b2);
        }
        zrow(K - 1, ec1, ec2);  // the centre row K
        float2 ra[M], rc[M];
        pr_rows_sum<K>(tb.pmass_fe, tb.pmass_fo, E2, O2, ec2, tb.plap_fe, tb.plap_fo, E1, O1, ec1, ra);
        pr_rows<K>(tb.pmass_fe, tb.pmass_fo, E1, O1, ec1, rc);
        if (act) {
          float2 *d1 = V1 + zi * S::VL.p + xx * S::VL.c, *d2 = V2 + zi * S::VL.p + xx * S::VL.c;
#pragma unroll
          for (int i = 0; i < M; ++i) {
            d1[i * S::VL.r] = ra[i];
            d2[i * S::VL.r] = rc[i];
          }
        }
      }
      team_sync();
    }
    // ---- x: r = b - s (M_x V1 + L_x V2), then S^T along x -> QA ----
#pragma unroll
    for (int j = 0; j < NPW; ++j) {
      const int t0 = lane + 32 * (wt + TEAM * j);
      const bool act = t0 < S::NQT;  // idle lanes redo task lane % NQT, stores skipped
      const int t = act ? t0 : lane % S::NQT;
      {
        const int zi = t / M, yi = t % M;
        float bv1[M], bv2[M];
        if constexpr (K % 4 == 0 && W % 4 == 0) {
          // the box origin is a multiple of 4 entries (x-offset 0): the row's
          // interior is entries 1..M of two 16-byte vectors per group of 4;
          // 8 lanes of rows 12 entries apart cover 32 distinct banks
          const float4 *r1 = reinterpret_cast<const float4 *>(bslA + (zi * M + yi) * W);
          const float4 *r2 = reinterpret_cast<const float4 *>(bslB + (zi * M + yi) * W);
#pragma unroll
          for (int g = 0; g < (M + 1) / 4; ++g) {
            const float4 u1 = r1[g], u2 = r2[g];
            const float e1[4] = {u1.x, u1.y, u1.z, u1.w}, e2[4] = {u2.x, u2.y, u2.z, u2.w};
#pragma unroll
            for (int c = 0; c < 4; ++c) {
              const int i = 4 * g + c - 1;
              if (i >= 0 && i < M) {
                bv1[i] = e1[c];
                bv2[i] = e2[c];
              }
            }
          }
        } else {
          const float *b1 = bslA + (zi * M + yi) * W + xoa + 1, *b2 = bslB + (zi * M + yi) * W + xob + 1;
#pragma unroll
          for (int i = 0; i < M; ++i) {
            bv1[i] = b1[i];
            bv2[i] = b2[i];
          }
        }
        float2 res[M];
        if (!a.zero_x) {
          const float2 *s1 = V1 + t, *s2 = V2 + t;  // = zi * VL.p + yi * VL.r
          float2 v[N1], E1[K], O1[K], ec1, E2[K], O2[K], ec2;
#pragma unroll
          for (int qq = 0; qq < N1; ++qq) v[qq] = s1[qq * S::VL.c];
          pr_fold<K>(v, E1, O1, ec1);
#pragma unroll
          for (int qq = 0; qq < N1; ++qq) v[qq] = s2[qq * S::VL.c];
          pr_fold<K>(v, E2, O2, ec2);
          float2 ra[M];
          pr_rows_sum<K>(tb.pmass_fe, tb.pmass_fo, E1, O1, ec1, tb.plap_fe, tb.plap_fo, E2, O2, ec2, ra);
#pragma unroll
          for (int i = 0; i < M; ++i) res[i] = pr_fma(-scale, ra[i], make_float2(bv1[i], bv2[i]));
        } else {
#pragma unroll
          for (int i = 0; i < M; ++i) res[i] = make_float2(bv1[i], bv2[i]);
        }
        float2 qv[M];
        pr_evec<K, true>(res, qv);
        float2 *d = QAb + zi * QA.p + yi * QA.r;
        if (act) {
#pragma unroll
          for (int i = 0; i < M; ++i) d[i * QA.c] = qv[i];
        }
      }
    }
    team_sync();
    // the staged boxes and slabs are consumed: fetch the next pair now
    if (tid == 0 && q + G < n_pairs) {
      fence_proxy_async_smem();
      issue(nxa, nya, nza, nxb, nyb, nzb);
    }
    // ---- the four fast-diagonalisation stages: each lane's tasks of this
    // warp's passes side by side (all loads, then the independent
    // contractions, then the stores), so their chains interleave ----
    int tq[NPW];
    bool aq[NPW];
#pragma unroll
    for (int j = 0; j < NPW; ++j) {
      const int t0 = lane + 32 * (wt + TEAM * j);
      aq[j] = t0 < S::NQT;  // idle lanes redo task lane % NQT, stores skipped
      tq[j] = aq[j] ? t0 : lane % S::NQT;
    }
    // ---- S^T along y: QA -> QB ----
    {
      float2 v[NPW][M], qv[NPW][M];
#pragma unroll
      for (int p = 0; p < NPW; ++p) {
        const float2 *src = QAb + (tq[p] / M) * QA.p + (tq[p] % M) * QA.c;
#pragma unroll
        for (int jj = 0; jj < M; ++jj) v[p][jj] = src[jj * QA.r];
      }
#pragma unroll
      for (int p = 0; p < NPW; ++p) pr_evec<K, true>(v[p], qv[p]);
#pragma unroll
      for (int p = 0; p < NPW; ++p) {
        float2 *d = QBb + (tq[p] / M) * QB.p + (tq[p] % M) * QB.c;
        if (aq[p]) {
#pragma unroll
          for (int jj = 0; jj < M; ++jj) d[jj * QB.r] = qv[p][jj];
        }
      }
    }
    team_sync();
    // ---- S^T along z, eigenvalue scaling, S along z: QB -> QC ----
    {
      float2 v[NPW][M], qv[NPW][M];
#pragma unroll
      for (int p = 0; p < NPW; ++p) {
        const float2 *src = QBb + (tq[p] / M) * QB.r + (tq[p] % M) * QB.c;
#pragma unroll
        for (int jj = 0; jj < M; ++jj) v[p][jj] = src[jj * QB.p];
      }
#pragma unroll
      for (int p = 0; p < NPW; ++p) {
        pr_evec<K, true>(v[p], qv[p]);
#pragma unroll
        for (int jj = 0; jj < M; ++jj) qv[p][jj] = pr_mul(rl[p][jj], qv[p][jj]);
        pr_evec<K, false>(qv[p], v[p]);
      }
#pragma unroll
      for (int p = 0; p < NPW; ++p) {
        float2 *d = QAb + (tq[p] / M) * QC.r + (tq[p] % M) * QC.c;
        if (aq[p]) {
#pragma unroll
          for (int jj = 0; jj < M; ++jj) d[jj * QC.p] = v[p][jj];
        }
      }
    }
    team_sync();
    // ---- S along x: QC -> QD ----
    {
      float2 v[NPW][M], qv[NPW][M];
#pragma unroll
      for (int p = 0; p < NPW; ++p) {
        const float2 *src = QAb + (tq[p] / M) * QC.p + (tq[p] % M) * QC.r;
#pragma unroll
        for (int jj = 0; jj < M; ++jj) v[p][jj] = src[jj * QC.c];
      }
#pragma unroll
      for (int p = 0; p < NPW; ++p) pr_evec<K, false>(v[p], qv[p]);
#pragma unroll
      for (int p = 0; p < NPW; ++p) {
        float2 *d = QBb + (tq[p] / M) * QD.p + (tq[p] % M) * QD.r;
        if (aq[p]) {
#pragma unroll
          for (int i = 0; i < M; ++i) d[i * QD.c] = qv[p][i];
        }
      }
    }
    team_sync();
    // ---- S along y and store x_I of both patches ----
    {
      float *const xpa = x + (fxa + 1 + (fya + 1) * a.sy + (fza + 1) * a.sz);
      float *const xpb = x + (fxb + 1 + (fyb + 1) * a.sy + (fzb + 1) * a.sz);
      const int sy32 = static_cast<int>(a.sy), sz32 = static_cast<int>(a.sz);
      float2 v[NPW][M], qv[NPW][M];
#pragma unroll
      for (int p = 0; p < NPW; ++p) {
        const float2 *src = QBb + (tq[p] / M) * QD.p + (tq[p] % M) * QD.c;
#pragma unroll
        for (int jj = 0; jj < M; ++jj) v[p][jj] = src[jj * QD.r];
      }
#pragma unroll
      for (int p = 0; p < NPW; ++p) pr_evec<K, false>(v[p], qv[p]);
#pragma unroll
      for (int p = 0; p < NPW; ++p) {
        const int o = tq[p] % M + (tq[p] / M) * sz32;
        if (aq[p]) {
#pragma unroll
          for (int jj = 0; jj < M; ++jj) xpa[o + jj * sy32] = qv[p][jj].x;
        }
        if (aq[p] && store_b) {
#pragma unroll
          for (int jj = 0; jj < M; ++jj) xpb[o + jj * sy32] = qv[p][jj].y;
        }
      }
    }
    team_sync();  // the Q buffers (inside the Z region) are read before the next z stage
    fxa = nxa;
    fya = nya;
    fza = nza;
    fxb = nxb;
    fyb = nyb;
    fzb = nzb;
  }
}

}  // namespace tps
