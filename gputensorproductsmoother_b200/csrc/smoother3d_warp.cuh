// 3D fused vertex-patch smoother with one warp per patch (sm_100a).
//
// Same per-patch algebra and contraction order as smoother3d_kernel (the
// reference's FUSED_CF patch kernel, include/loop_kernel.cuh:962-1060 with
// include/evaluate_kernel.cuh:501-590, 1327-1434, 2058-2163): the box residual
// b - A x~ with the interior of x set to zero (z: M, L -> y: 3 products ->
// x: 2 products), then the fast-diagonalisation solve S^T_x, S^T_y, S^T_z,
// scaling, S_z, S_x, S_y and the store of omega A_II^{-1} r_I.  The
// arithmetic of a patch is the same operation for operation, so both
// kernels give bit-identical sweeps.
//
// Execution model: a team of warps -- one CTA; two warps in FP64 from degree
// 4 on, where every stage has at least two 32-lane passes -- owns its patches, one
// shared-memory stage and one mbarrier; warp w of the team takes passes w,
// w + TEAM, ... of every stage, so twice the warps per SM share the stage's
// shared memory.  The seven contraction stages of a patch are separated by
// the team's barrier (the warp's own __syncwarp for a one-warp team); teams
// never wait for one another (a CTA-wide batch of patches loses about half
// of its issue slots at the barriers between stages).  The next patch's x box
// and b slab are fetched by TMA as soon as the x stage has consumed the
// current ones, so the load overlaps the four fast-diagonalisation stages of
// the same team and the work of the other teams on the SM.
//
// Shared-memory strides: each staged array is written by one stage and read
// by the next with a fixed lane -> line mapping (y stage: zi = t % M,
// xx = t / M; every other stage: (a, b) = (t / M, t % M) over its two line
// coordinates).  The strides below were chosen by an exhaustive search over
// padded strides so that these warp-wide accesses hit each bank once where
// possible (every fast-diagonalisation access) and at most twice elsewhere,
// at a few percent more shared memory than the dense layout.
#pragma once

#include <cuda.h>

#include "ptx.cuh"
#include "smoother3d.cuh"
#include "tps_common.cuh"

namespace tps {

struct Str3 {
  int p, r, c;  // strides of the (z, y, x) indices
};

// strides of Z1/Z2 [zi][y][x] (RZ, PZ), V1/V2 [zi][yi][x] (RV, PV) and the
// four fast-diagonalisation arrays; the primary template is the dense layout
template <int K, int ES>
struct WpLayout {
  static constexpr int N1 = 2 * K + 1, M = 2 * K - 1;
  static constexpr int RZ = N1, PZ = N1 * N1, RV = N1, PV = M * N1;
  static constexpr Str3 QA{M * M, M, 1}, QB{M * M, M, 1}, QC{M * M, M, 1}, QD{M * M, M, 1};
};
template <>
struct WpLayout<2, 4> {
  static constexpr int RZ = 5, PZ = 25, RV = 5, PV = 19;
  static constexpr Str3 QA{1, 3, 9}, QB{1, 3, 9}, QC{1, 3, 9}, QD{1, 3, 9};
};
template <>
struct WpLayout<3, 4> {
  static constexpr int RZ = 7, PZ = 50, RV = 9, PV = 45;
  static constexpr Str3 QA{5, 1, 25}, QB{1, 25, 5}, QC{1, 5, 25}, QD{5, 1, 25};
};
template <>
struct WpLayout<4, 4> {
  static constexpr int RZ = 9, PZ = 87, RV = 9, PV = 67;
  static constexpr Str3 QA{7, 1, 65}, QB{7, 71, 1}, QC{7, 1, 55}, QD{7, 1, 65};
};
template <>
struct WpLayout<5, 4> {
  static constexpr int RZ = 11, PZ = 121, RV = 11, PV = 99;
  static constexpr Str3 QA{9, 1, 97}, QB{9, 105, 1}, QC{9, 1, 89}, QD{9, 1, 97};
};
template <>
struct WpLayout<2, 8> {
  static constexpr int RZ = 5, PZ = 27, RV = 7, PV = 21;
  static constexpr Str3 QA{3, 1, 9}, QB{1, 9, 3}, QC{1, 3, 9}, QD{3, 1, 9};
};
template <>
struct WpLayout<3, 8> {
  static constexpr int RZ = 7, PZ = 50, RV = 7, PV = 35;
  static constexpr Str3 QA{5, 1, 33}, QB{5, 37, 1}, QC{25, 5, 1}, QD{5, 1, 33};
};
template <>
struct WpLayout<4, 8> {
  static constexpr int RZ = 9, PZ = 87, RV = 9, PV = 63;
  static constexpr Str3 QA{7, 1, 49}, QB{7, 55, 1}, QC{1, 7, 49}, QD{7, 1, 49};
};

// degrees and precisions with a compiled warp-per-patch kernel (larger
// patches leave too few warps per SM: their stage alone exceeds 20 KB)
template <int K, typename T>
constexpr bool wp3_enabled()
{
  return K >= 2 && (sizeof(T) == 4 ? K <= 5 : K <= 4);
}

constexpr int wp_max(int a, int b) { return a > b ? a : b; }
constexpr int wp_rup(int a, int m) { return (a + m - 1) / m * m; }

template <int K, typename T, int TEAM>
struct Wp3 {
  using L = WpLayout<K, static_cast<int>(sizeof(T))>;
  static constexpr int N1 = 2 * K + 1, M = 2 * K - 1;
  static constexpr int A = Sm3<K, T>::A, W = Sm3<K, T>::W;  // the TMA boxes of the shared views
  static constexpr int XBOX = N1 * N1 * W, BBOX = M * M * W;
  static constexpr int ALIGN = 128 / static_cast<int>(sizeof(T));
  static constexpr int ZEXT = (M - 1) * L::PZ + (N1 - 1) * L::RZ + N1;
  static constexpr int VEXT = (M - 1) * L::PV + (M - 1) * L::RV + N1;
  static constexpr int ext(Str3 s) { return (M - 1) * (s.p + s.r + s.c) + 1; }
  static constexpr int QBUF1 = wp_max(ext(L::QA), ext(L::QC)), QBUF2 = wp_max(ext(L::QB), ext(L::QD));
  // per team: [x box, later V1 | V2] [b slab] [Z1 | Z2, later QA/QC | QB/QD]
  static constexpr int BOFF = wp_rup(wp_max(XBOX, 2 * VEXT), ALIGN);
  static constexpr int ZOFF = BOFF + BBOX;
  static constexpr int WARP_ELEMS = wp_rup(ZOFF + wp_max(2 * ZEXT, QBUF1 + QBUF2), ALIGN);
  static constexpr int NT = 32 * TEAM;  // one team = one CTA, one patch at a time
  // the eigenvalue scalings live in registers (no shared table), so that the
  // stage alone sets the CTAs per SM
  static constexpr size_t OFF_BAR = sizeof(T) * static_cast<size_t>(WARP_ELEMS);
  static constexpr size_t BYTES = OFF_BAR + 8;
  // line tasks of the stages and their 32-lane passes per warp of the team
  static constexpr int RING = N1 * N1 - M * M, IPAIR = (M * M + 1) / 2;
  static constexpr int NZT = RING + IPAIR, NYT = M * N1, NQT = M * M;
  static constexpr int NZP = (NZT + 31) / 32, NYP = (NYT + 31) / 32, NQP = (NQT + 31) / 32;
  static constexpr int NZPW = (NZP + TEAM - 1) / TEAM, NYPW = (NYP + TEAM - 1) / TEAM;
  static constexpr int NQPW = (NQP + TEAM - 1) / TEAM;
};

// warps per patch (the team, one CTA): two in FP64 from degree 4 on, one
// otherwise (measured at 3D Q4, ms per sweep, one warp vs two: FP64 64^3
// 1.053 vs 0.998, 32^3 0.152 vs 0.148; FP32 64^3 0.564 vs 0.604, where the
// pair kernel is the default anyway)
template <int K, typename T>
constexpr int wp3_warps()
{
  return K >= 4 && sizeof(T) == 8 ? 2 : 1;
}

// CTAs per SM (the register budget of __launch_bounds__): as many as shared
// memory holds (228 KB, 1 KB reserved per CTA, at most 32 CTAs), at most 32
// warps per SM for the FP64 degree-4 teams and 18 otherwise (10 CTAs of the
// FP64 degree-4 team fit, about 76 registers a thread)
template <int K, typename T>
constexpr int wp3_ctas()
{
  constexpr int w = wp3_warps<K, T>();
  constexpr int max_warps = w == 2 && K <= 4 ? 32 : 18;
  int c = static_cast<int>(233472 / (Wp3<K, T, w>::BYTES + 1024));
  if (c * w > max_warps) c = max_warps / w;
  return c > 32 ? 32 : c < 1 ? 1 : c;
}

// patch lattice index -> box origin (first DoF coordinates), divisions as
// multiply-shifts
__device__ __forceinline__ void wp_patch_xyz(const Sm3Args &a, int j, int k, int &fx, int &fy, int &fz)
{
  const int jz = fast_div(j, a.mxy, a.sxy), rz = j - jz * (a.nx_c * a.ny_c);
  const int jy = fast_div(rz, a.mx, a.sx), jx = rz - jy * a.nx_c;
  fx = (a.cx + 2 * jx) * k;
  fy = (a.cy + 2 * jy) * k;
  fz = (a.cz + 2 * jz) * k;
}

template <int K, typename T, int TEAM>
__global__ void __launch_bounds__(32 * TEAM, wp3_ctas<K, T>())
    smoother3d_warp_kernel(const __grid_constant__ CUtensorMap map_x, const __grid_constant__ CUtensorMap map_b,
                           T *__restrict__ x, const Sm3Args a, T scale, T fd_scale, int *__restrict__ err)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  using S = Wp3<K, T, TEAM>;
  using Lo = typename S::L;
  using P2 = typename Pair<T>::type;
  constexpr int N1 = S::N1, M = S::M, W = S::W, AL = S::A;
  constexpr Str3 QA = Lo::QA, QB = Lo::QB, QC = Lo::QC, QD = Lo::QD;
  const DegreeTables<K, T> &tb = c_tables<K, T>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int tid = threadIdx.x, lane = tid & 31, wt = tid >> 5;  // wt: warp within the team
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw + S::OFF_BAR);
  T *stage = reinterpret_cast<T *>(smem_raw);
  // the team's barrier between stages (one warp: the warp's own)
  auto team_sync = [&]() {
    if constexpr (TEAM == 1)
      __syncwarp();
    else
      __syncthreads();
  };
  T *Z1 = stage + S::ZOFF, *Z2 = Z1 + S::ZEXT;
  T *V1 = stage, *V2 = stage + S::VEXT;
  T *QAb = Z1, *QBb = Z1 + S::QBUF1;  // QA and QC share one buffer, QB and QD the other
  const T *bsl = stage + S::BOFF;

  // fd_scale / (lambda_x + lambda_y + lambda_z) for this lane's lines of the
  // z stage of the solve (t = (y mode, x mode) = (t / M, t % M), one per
  // pass of this warp) and every z mode, kept in registers
  T rl[S::NQPW][M];
#pragma unroll
  for (int jp = 0; jp < S::NQPW; ++jp) {
    const int t0 = lane + 32 * (wt + TEAM * jp);
    const int t = t0 < S::NQT ? t0 : 0;  // lanes without a line compute an unused value
    const T exy = tb.eval[t % M], eyy = tb.eval[t / M];
#pragma unroll
    for (int jj = 0; jj < M; ++jj) rl[jp][jj] = fd_scale / (exy + eyy + tb.eval[jj]);
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  __syncthreads();  // the mbarrier is ready

  const int G = gridDim.x;
  int j = blockIdx.x;
  auto issue = [&](int fx, int fy, int fz) {  // thread 0: the x box and b slab of the patch at (fx, fy, fz)
    const int x0 = fx & ~(AL - 1);
    mbar_arrive_expect_tx(bar, static_cast<uint32_t>(sizeof(T) * (S::BBOX + (a.zero_x ? 0 : S::XBOX))));
    if (!a.zero_x) tma_load_3d(stage, &map_x, bar, x0, fy, fz);
    tma_load_3d(stage + S::BOFF, &map_b, bar, x0, fy + 1, fz + 1);
  };
  int fx = 0, fy = 0, fz = 0;
  if (j < a.n_patches) {
    wp_patch_xyz(a, j, K, fx, fy, fz);
    if (tid == 0) issue(fx, fy, fz);
  }

  for (int it = 0; j < a.n_patches; j += G, ++it) {
    const int xo = fx & (AL - 1);
    int nfx = 0, nfy = 0, nfz = 0;  // the next patch of this team
    if (j + G < a.n_patches) wp_patch_xyz(a, j + G, K, nfx, nfy, nfz);
    const bool ok = mbar_wait_bounded(bar, it & 1);
    if (TEAM == 1 ? !__all_sync(0xffffffffu, ok) : !__syncthreads_and(ok)) {
      if (tid == 0) atomicExch(err, 1);
      return;  // the only copy in flight was the one waited for
    }

    if (!a.zero_x) {
      // ---- z: Z1 = M_z x~, Z2 = L_z x~ (ring lines, then pairs of interior lines) ----
      const T *box = stage + xo;
#pragma unroll
      for (int jp = 0; jp < S::NZPW; ++jp) {
        const int t = lane + 32 * (wt + TEAM * jp);
        if (t < S::RING) {
          int y, xx;
          if (t < N1) {
            y = 0;
            xx = t;
          } else if (t < 2 * N1) {
            y = N1 - 1;
            xx = t - N1;
          } else {
            const int q = t - 2 * N1;
            y = 1 + (q >> 1);
            xx = (q & 1) ? N1 - 1 : 0;
          }
          const T *src = box + y * W + xx;
          T v[N1], ec, r1[M], r2[M];
          P2 eo[K > 1 ? K : 1];
#pragma unroll
          for (int z = 0; z < N1; ++z) v[z] = src[z * N1 * W];
          fold_pairs<K, T>(v, eo, ec);
          rows_mass<K, T>(eo, ec, r1);
          rows_lap<K, T>(eo, ec, r2);
          T *d1 = Z1 + y * Lo::RZ + xx, *d2 = Z2 + y * Lo::RZ + xx;
#pragma unroll
          for (int i = 0; i < M; ++i) {
            d1[i * Lo::PZ] = r1[i];
            d2[i * Lo::PZ] = r2[i];
          }
        } else if (t < S::NZT) {
          const int r0 = 2 * (t - S::RING);
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int r = r0 + h;
            if (r < M * M) {
              const int y = 1 + r / M, xx = 1 + r % M;
              const T *src = box + y * W + xx;
              const T v0 = src[0], vn = src[(N1 - 1) * N1 * W];
              T *d1 = Z1 + y * Lo::RZ + xx, *d2 = Z2 + y * Lo::RZ + xx;
#pragma unroll
              for (int i = 0; i < M; ++i) {
                d1[i * Lo::PZ] = fmadd(tb.pmass[(i + 1) * N1 + N1 - 1], vn, tb.pmass[(i + 1) * N1] * v0);
                d2[i * Lo::PZ] = fmadd(tb.plap[(i + 1) * N1 + N1 - 1], vn, tb.plap[(i + 1) * N1] * v0);
              }
            }
          }
        }
      }
      team_sync();
      // ---- y: V1 = M_y Z2 + L_y Z1, V2 = M_y Z1 (V overwrites the dead x box) ----
#pragma unroll
      for (int jp = 0; jp < S::NYPW; ++jp) {
        const int t = lane + 32 * (wt + TEAM * jp);
        if (t < S::NYT) {
          const int zi = t % M, xx = t / M;
          const T *s1 = Z1 + zi * Lo::PZ + xx, *s2 = Z2 + zi * Lo::PZ + xx;
          T v[N1], ec1, ec2;
          P2 eo1[K > 1 ? K : 1], eo2[K > 1 ? K : 1];
#pragma unroll
          for (int q = 0; q < N1; ++q) v[q] = s1[q * Lo::RZ];
          fold_pairs<K, T>(v, eo1, ec1);
#pragma unroll
          for (int q = 0; q < N1; ++q) v[q] = s2[q * Lo::RZ];
          fold_pairs<K, T>(v, eo2, ec2);
          T ra[M], rc[M];
          rows_mass_lap<K, T>(eo2, ec2, eo1, ec1, ra);
          rows_mass<K, T>(eo1, ec1, rc);
          T *d1 = V1 + zi * Lo::PV + xx, *d2 = V2 + zi * Lo::PV + xx;
#pragma unroll
          for (int i = 0; i < M; ++i) {
            d1[i * Lo::RV] = ra[i];
            d2[i * Lo::RV] = rc[i];
          }
        }
      }
      team_sync();
    }
    // ---- x: r = b - s (M_x V1 + L_x V2), then S^T along x -> QA ----
#pragma unroll
    for (int jp = 0; jp < S::NQPW; ++jp) {
      const int t = lane + 32 * (wt + TEAM * jp);
      if (t < S::NQT) {
        const int zi = t / M, yi = t % M;
        const T *bb = bsl + (zi * M + yi) * W + xo + 1;
        T res[M];
        if (!a.zero_x) {
          const T *s1 = V1 + zi * Lo::PV + yi * Lo::RV, *s2 = V2 + zi * Lo::PV + yi * Lo::RV;
          T v[N1], ec1, ec2;
          P2 eo1[K > 1 ? K : 1], eo2[K > 1 ? K : 1];
#pragma unroll
          for (int q = 0; q < N1; ++q) v[q] = s1[q];
          fold_pairs<K, T>(v, eo1, ec1);
#pragma unroll
          for (int q = 0; q < N1; ++q) v[q] = s2[q];
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
        T *d = QAb + zi * QA.p + yi * QA.r;
#pragma unroll
        for (int i = 0; i < M; ++i) d[i * QA.c] = q[i];
      }
    }
    team_sync();
    // the staged box and slab are consumed: fetch the next patch now
    if (tid == 0 && j + G < a.n_patches) {
      fence_proxy_async_smem();
      issue(nfx, nfy, nfz);
    }
    // ---- S^T along y: QA -> QB ----
#pragma unroll
    for (int jp = 0; jp < S::NQPW; ++jp) {
      const int t = lane + 32 * (wt + TEAM * jp);
      if (t < S::NQT) {
        const int zi = t / M, qx = t % M;
        const T *s = QAb + zi * QA.p + qx * QA.c;
        T v[M], q[M];
#pragma unroll
        for (int jj = 0; jj < M; ++jj) v[jj] = s[jj * QA.r];
        evec_apply<K, T, true>(v, q);
        T *d = QBb + zi * QB.p + qx * QB.c;
#pragma unroll
        for (int jj = 0; jj < M; ++jj) d[jj * QB.r] = q[jj];
      }
    }
    team_sync();
    // ---- S^T along z, eigenvalue scaling, S along z: QB -> QC ----
#pragma unroll
    for (int jp = 0; jp < S::NQPW; ++jp) {
      const int t = lane + 32 * (wt + TEAM * jp);
      if (t < S::NQT) {
        const int yi = t / M, xi = t % M;
        const T *s = QBb + yi * QB.r + xi * QB.c;
        T v[M], q[M];
#pragma unroll
        for (int jj = 0; jj < M; ++jj) v[jj] = s[jj * QB.p];
        evec_apply<K, T, true>(v, q);
#pragma unroll
        for (int jj = 0; jj < M; ++jj) q[jj] *= rl[jp][jj];
        evec_apply<K, T, false>(q, v);
        T *d = QAb + yi * QC.r + xi * QC.c;
#pragma unroll
        for (int jj = 0; jj < M; ++jj) d[jj * QC.p] = v[jj];
      }
    }
    team_sync();
    // ---- S along x: QC -> QD ----
#pragma unroll
    for (int jp = 0; jp < S::NQPW; ++jp) {
      const int t = lane + 32 * (wt + TEAM * jp);
      if (t < S::NQT) {
        const int zi = t / M, yi = t % M;
        const T *s = QAb + zi * QC.p + yi * QC.r;
        T v[M], q[M];
#pragma unroll
        for (int jj = 0; jj < M; ++jj) v[jj] = s[jj * QC.c];
        evec_apply<K, T, false>(v, q);
        T *d = QBb + zi * QD.p + yi * QD.r;
#pragma unroll
        for (int i = 0; i < M; ++i) d[i * QD.c] = q[i];
      }
    }
    team_sync();
    // ---- S along y and store x_I ----
    // 64-bit patch base once; 32-bit offsets within the patch (a patch spans
    // less than 2 planes of a level of < 2^31 entries)
    T *const xp = x + (fx + 1 + (fy + 1) * a.sy + (fz + 1) * a.sz);
    const int sy32 = static_cast<int>(a.sy), sz32 = static_cast<int>(a.sz);
#pragma unroll
    for (int jp = 0; jp < S::NQPW; ++jp) {
      const int t = lane + 32 * (wt + TEAM * jp);
      if (t < S::NQT) {
        const int z = t / M, xx = t % M;
        const T *s = QBb + z * QD.p + xx * QD.c;
        T v[M], q[M];
#pragma unroll
        for (int jj = 0; jj < M; ++jj) v[jj] = s[jj * QD.r];
        evec_apply<K, T, false>(v, q);
        const int o = xx + z * sz32;
#pragma unroll
        for (int jj = 0; jj < M; ++jj) xp[o + jj * sy32] = q[jj];
      }
    }
    team_sync();  // the Q buffers (inside the Z region) are read before the next z stage
    fx = nfx;
    fy = nfy;
    fz = nfz;
  }
}

}  // namespace tps
