// 3D vertex-patch smoother on the 5th-generation tensor cores (sm_100a).
//
// The colour step of smoother3d_kernel (reference: loop_kernel_fused_cf +
// LocalSmoother<FUSED_CF>, include/loop_kernel.cuh:962-1060,
// include/evaluate_kernel.cuh:501-590, 1327-1434, 2058-2163) in the ring form
//     x_I <- omega A_II^{-1} (b_I - A_IB x_B),
// with every 1D contraction of a patch issued as a tcgen05.mma of kind::tf32
// (TF32 operands from shared memory, FP32 accumulation in tensor memory).
// The lines of the patch along the contracted direction are the MMA rows
// (M = 128), the 1D matrix is the B operand (K = entries of a line, N =
// outputs); both operands are K-major.  Nine MMA stages per patch:
//   S1  x: [M_x | L_x] on the x box whose interior has been set to zero
//   S2  y: V1 = M_y X2 + L_y X1, V2 = M_y X1
//   S3  z: -s (M_z V1 + L_z V2); the epilogue adds b: the residual r
//   S4  S^T_z    S5  S^T_y    S6  S^T_x, then 1/(lambda sums) in registers
//   S7  S_x      S8  S_y      S9  S_z, stored to global memory
// Between two stages every thread of the warpgroup takes one TMEM lane (one
// line) with tcgen05.ld and writes it to shared memory in the operand layout
// of the next stage, which contracts another direction, rounded to the
// nearest TF32 value (cvt.rna; the tensor cores would otherwise truncate,
// and truncation biases the sweep: about 6e-3 instead of 9e-4 relative
// deviation from an FP64 sweep at degree 4).
//
// Work split: a "unit" is one warpgroup (4 warps = the 128 TMEM lanes) that
// solves one patch at a time; U units per CTA, persistent CTAs.  A unit owns
// two slots, the patch being solved and the prefetch of its next patch.  TMA
// stages the x box directly in the K-major operand layout of S1: rank-4 boxes
// (x%4, 8 rows of y, x/4, z) land as [z][x/4][y%8][x%4], i.e. 8-row groups
// (one per z and 8 rows of y) of 16-byte chunks of x; the b interior comes
// as a plain [z][y][x] box.  The 1D matrices of all stages are built once
// per CTA from the constant tables (rounded to TF32).
//
// Operand padding: MMA rows past a patch's lines and K entries past a line's
// length read neighbouring shared memory, which holds finite values (the
// whole allocation is zeroed first and only finite data are written); the
// matching B entries are zero and the extra D rows are never read.
#pragma once

#include <cuda.h>

#include "ptx.cuh"
#include "smoother3d.cuh"
#include "tps_common.cuh"

namespace tps {

template <int K>
struct Tc3 {
  static constexpr int cdiv(int a, int b) { return (a + b - 1) / b; }
  static constexpr int rup(int a, int b) { return cdiv(a, b) * b; }
  static constexpr int mx(int a, int b) { return a > b ? a : b; }
  static constexpr int N1 = 2 * K + 1, M = 2 * K - 1;
  // largest x offset of a patch box inside its 16-byte aligned TMA box
  static constexpr int XO = K % 4 == 0 ? 0 : (K % 2 == 0 ? 2 : 3);
  static constexpr int XC = cdiv(XO + N1, 4), XW = 4 * XC;  // 16-byte chunks per staged row
  // S1: row y%8 + 8*(z + N1*(y/8)), K = box x; groups of 8 rows at SBO1
  static constexpr int YH = cdiv(N1, 8), R1 = 8 * N1 * YH, T1 = cdiv(R1, 128);
  static constexpr int K1 = rup(XW, 8), KS1 = K1 / 8, NB1 = rup(2 * M, 16);
  static constexpr int SBO1 = XC * 128;
  static constexpr int XBOX = YH * N1 * SBO1;  // YH TMA loads of N1 groups
  // S2: row xi + M*z, K = 2y + (0: X1, 1: X2)
  static constexpr int R2 = M * N1, T2 = cdiv(R2, 128), K2 = rup(2 * N1, 8), KS2 = K2 / 8;
  static constexpr int NB2 = rup(2 * M, 16), SBO2 = (K2 / 4) * 128 + 16;
  static constexpr int A2 = cdiv(R2, 8) * SBO2;
  // S3: row xi + M*yi, K = 2z + (0: V1, 1: V2)
  static constexpr int R3 = M * M, T3 = cdiv(R3, 128), K3 = rup(2 * N1, 8), KS3 = K3 / 8;
  static constexpr int NB3 = rup(M, 16), SBO3 = (K3 / 4) * 128 + 16;
  static constexpr int A3 = cdiv(R3, 8) * SBO3;
  // S4..S9: row a + M*b over the M^2 lines, K = contracted index
  static constexpr int RF = M * M, TF = cdiv(RF, 128), KF = rup(M, 8), KSF = KF / 8;
  static constexpr int NBF = rup(M, 16), SBOF = (KF / 4) * 128 + 16;
  static constexpr int AF = cdiv(RF, 8) * SBOF;
  static constexpr int BBOX = M * M * XW * 4;  // b interior, [zi][yi][box x]
  // one slot: work region (x box, then the operands of S2..S9) + b box.
  // Two slots per unit (the patch being solved and the TMA prefetch of its
  // next patch) up to degree 4; one from degree 5 on, where a slot is 17-40 KB
  // and the units that fit instead (8, 7 and 5 per SM at degrees 5, 6 and 7
  // against 6, 3 and 2 with prefetch slots) overlap one another's stages
  static constexpr int WORK = rup(mx(mx(XBOX, A2), mx(A3, AF)), 128);
  static constexpr int SLOT = WORK + rup(BBOX, 128);
  static constexpr int SLOTS = K >= 5 ? 1 : 2;
  static constexpr int UNIT = SLOTS * SLOT;
  static constexpr int COLS = mx(mx(T1 * NB1, T2 * NB2), mx(T3 * NB3, TF * NBF));  // TMEM columns
  // furthest byte an MMA may read, relative to its slot (16 groups of 8 rows per tile)
  static constexpr int EXT = mx(mx(T1 * 16 * SBO1 + KS1 * 256, T2 * 16 * SBO2 + KS2 * 256),
                                mx(T3 * 16 * SBO3 + KS3 * 256, TF * 16 * SBOF + KSF * 256));
  static constexpr int SLACK = EXT > SLOT ? rup(EXT - SLOT, 128) : 0;
  // per-CTA B matrices (K-major: 8-row groups of KB/4 chunks of 128 bytes)
  static constexpr int NXO = XO + 1;
  static constexpr int SB1 = NB1 * K1 * 4, SB2 = NB2 * K2 * 4, SB3 = NB3 * K3 * 4, SBF = NBF * KF * 4;
  static constexpr int OFF_B1 = 0, OFF_B2 = OFF_B1 + NXO * SB1, OFF_B3 = OFF_B2 + SB2;
  static constexpr int OFF_BST = OFF_B3 + SB3, OFF_BS = OFF_BST + SBF, OFF_RL = OFF_BS + SBF;
  static constexpr int OFF_BAR = rup(OFF_RL + 4 * M * M * M, 128);  // 3 mbarriers per unit, TMEM base, abort flags
  static constexpr int OFF_UNITS = rup(OFF_BAR + 256, 1024);
  static constexpr int bytes_for(int u) { return OFF_UNITS + u * UNIT + SLACK; }
  static constexpr int tmem_cols(int u)
  {
    return u * COLS <= 32 ? 32 : u * COLS <= 64 ? 64 : u * COLS <= 128 ? 128 : u * COLS <= 256 ? 256 : 512;
  }
  // CTAs per SM for u units per CTA: shared memory (+1 KB reserved per CTA),
  // tensor memory, and at most 10 warpgroups per SM (48 registers a thread)
  static constexpr int per_sm(int u)
  {
    const int by_smem = 233472 / (bytes_for(u) + 1024), by_regs = 10 / u, by_tmem = 512 / tmem_cols(u);
    const int m = by_smem < by_regs ? by_smem : by_regs;
    return m < by_tmem ? m : by_tmem;
  }
  // units per CTA: the most units per SM, ties to the larger CTA
  static constexpr int pick_u()
  {
    int best = 0, bu = 0;
    for (int u = 1; u <= 8; ++u)
      if (bytes_for(u) <= 232448 && u * per_sm(u) >= best && per_sm(u) >= 1) {
        best = u * per_sm(u);
        bu = u;
      }
    return bu;
  }
  static constexpr int U = pick_u();
  static constexpr int NT = 128 * U;
  static constexpr int MINB = per_sm(U);  // CTAs per SM the registers must allow
  static constexpr int BYTES = bytes_for(U);
  static constexpr int TMEM_COLS = tmem_cols(U);
  static_assert(K >= 2 && K <= 7, "tensor-core smoother: degrees 2..7");
  static_assert(U >= 1, "tensor-core smoother: one unit must fit");
  static_assert((N1 * SBO1) % 128 == 0 && WORK % 128 == 0, "TMA destinations are 128-byte aligned");
};

// byte offset of element (m, k) of a K-major (no swizzle) TF32 operand:
// 8-row groups at stride sbo, rows 16 bytes apart, 4-entry K chunks at 128 bytes
__device__ __forceinline__ int km_off(int m, int k, int sbo)
{
  return (m >> 3) * sbo + ((m & 7) << 4) + ((k >> 2) << 7) + ((k & 3) << 2);
}

template <int K>
__global__ void __launch_bounds__(Tc3<K>::NT, Tc3<K>::MINB)
    smoother3d_tc_kernel(const __grid_constant__ CUtensorMap map_x, const __grid_constant__ CUtensorMap map_b,
                         float *__restrict__ x, const Sm3Args a, float scale, float fd_scale,
                         int *__restrict__ err)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  using C = Tc3<K>;
  constexpr int N1 = C::N1, M = C::M, U = C::U, NT = C::NT;
  const DegreeTables<K, float> &tb = c_tables<K, float>;
  extern __shared__ __align__(1024) unsigned char smem[];
  const int tid = threadIdx.x;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + C::OFF_BAR);
  uint32_t *s_tmem = reinterpret_cast<uint32_t *>(smem + C::OFF_BAR + 8 * 3 * U);
  int *s_abort = reinterpret_cast<int *>(smem + C::OFF_BAR + 8 * 3 * U + 16);
  float *RL = reinterpret_cast<float *>(smem + C::OFF_RL);

  // ---- prologue: zero the allocation, build the B operands -----------------
  for (int i = tid; i < C::BYTES / 16; i += NT) reinterpret_cast<uint4 *>(smem)[i] = make_uint4(0, 0, 0, 0);
  __syncthreads();
  auto bk = [&](int off, int kb, int n, int k) -> float & {
    return *reinterpret_cast<float *>(smem + off + (n >> 3) * (kb / 4) * 128 + ((n & 7) << 4) +
                                      ((k >> 2) << 7) + ((k & 3) << 2));
  };
  // S1 (one copy per box offset xo): n < M mass rows 1..M, M <= n < 2M
  // stiffness rows, K = box x (patch x = box x - xo)
  for (int e = tid; e < C::NXO * C::NB1 * C::K1; e += NT) {
    const int xo = e / (C::NB1 * C::K1), r = e % (C::NB1 * C::K1), n = r / C::K1, k = r % C::K1;
    const int xl = k - xo;
    float v = 0.f;
    if (xl >= 0 && xl < N1)
      v = n < M ? tb.pmass[(n + 1) * N1 + xl] : n < 2 * M ? tb.plap[(n - M + 1) * N1 + xl] : 0.f;
    bk(C::OFF_B1 + xo * C::SB1, C::K1, n, k) = to_tf32(v);
  }
  // S2: K = 2y + s; V1 = M_y X2 + L_y X1 (n < M), V2 = M_y X1 (M <= n < 2M)
  for (int e = tid; e < C::NB2 * C::K2; e += NT) {
    const int n = e / C::K2, k = e % C::K2, y = k >> 1, s = k & 1;
    float v = 0.f;
    if (y < N1) {
      if (n < M) v = s == 0 ? tb.plap[(n + 1) * N1 + y] : tb.pmass[(n + 1) * N1 + y];
      else if (n < 2 * M && s == 0) v = tb.pmass[(n - M + 1) * N1 + y];
    }
    bk(C::OFF_B2, C::K2, n, k) = to_tf32(v);
  }
  // S3: K = 2z + s; -scale (M_z V1 + L_z V2)
  for (int e = tid; e < C::NB3 * C::K3; e += NT) {
    const int n = e / C::K3, k = e % C::K3, z = k >> 1, s = k & 1;
    float v = 0.f;
    if (n < M && z < N1) v = -scale * (s == 0 ? tb.pmass[(n + 1) * N1 + z] : tb.plap[(n + 1) * N1 + z]);
    bk(C::OFF_B3, C::K3, n, k) = to_tf32(v);
  }
  // S^T (nodal k -> mode n) and S (mode k -> nodal n)
  for (int e = tid; e < C::NBF * C::KF; e += NT) {
    const int n = e / C::KF, k = e % C::KF;
    const bool in = n < M && k < M;
    bk(C::OFF_BST, C::KF, n, k) = to_tf32(in ? tb.evec[k * M + n] : 0.f);
    bk(C::OFF_BS, C::KF, n, k) = to_tf32(in ? tb.evec[n * M + k] : 0.f);
  }
  for (int e = tid; e < M * M * M; e += NT)
    RL[e] = fd_scale / (tb.eval[e % M] + tb.eval[(e / M) % M] + tb.eval[e / (M * M)]);
  if (tid < U) {
    mbar_init(&bars[3 * tid + 0], 1);
    mbar_init(&bars[3 * tid + 1], 1);
    mbar_init(&bars[3 * tid + 2], 1);
    s_abort[tid] = 0;
  }
  if (tid == 0) fence_mbar_init();
  if (tid < 32) tmem_alloc(s_tmem, C::TMEM_COLS);
  fence_proxy_async_smem();  // the B operands are read by the tensor cores
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;

  // ---- unit loop -------------------------------------------------------------
  const int u = tid >> 7, ut = tid & 127, wq = ut >> 5;
  const bool leader = ut == 0;
  unsigned char *slots = smem + C::OFF_UNITS + u * C::UNIT;
  uint64_t *tbar = bars + 3 * u, *mbar = bars + 3 * u + 2;
  const uint32_t tcol = tmem + u * C::COLS;                            // D base (lane 0)
  const uint32_t tme = tcol + (static_cast<uint32_t>(32 * wq) << 16);  // this warp's lanes
  const uint32_t s_base = smem_u32(smem);
  const int gstride = gridDim.x * U;
  uint32_t mph = 0;

  auto patch_xyz = [&](int j, int &fx, int &fy, int &fz) {
    const int jx = j % a.nx_c, jy = (j / a.nx_c) % a.ny_c, jz = j / (a.nx_c * a.ny_c);
    fx = (a.cx + 2 * jx) * K;
    fy = (a.cy + 2 * jy) * K;
    fz = (a.cz + 2 * jz) * K;
  };
  auto issue = [&](int pp, int sl) {
    unsigned char *w = slots + sl * C::SLOT, *bb = w + C::WORK;
    int fx, fy, fz;
    patch_xyz(pp, fx, fy, fz);
    const int x0 = fx & ~3;
    mbar_arrive_expect_tx(&tbar[sl], C::BBOX + (a.zero_x ? 0 : C::XBOX));
    if (!a.zero_x) {
#pragma unroll
      for (int yh = 0; yh < C::YH; ++yh) tma_load_4d(w + yh * N1 * C::SBO1, &map_x, &tbar[sl], 0, fy + 8 * yh, x0 >> 2, fz);
    }
    tma_load_3d(bb, &map_b, &tbar[sl], x0, fy + 1, fz + 1);
  };
  // every thread waits for the stage's MMAs (bounded); a timeout is recorded
  auto wait_mma = [&]() {
    if (!mbar_wait_bounded(mbar, mph)) {
      atomicExch(err, 1);
      s_abort[u] = 1;
    }
    mph ^= 1;
    tc_fence_after();
  };
  // make this thread's operand stores visible to the tensor cores, then sync the unit
  auto stage_sync = [&]() {
    fence_proxy_async_smem();
    tc_fence_before();
    named_bar(1 + u, 128);
  };
  // one stage: T tiles (16 groups of 8 rows each) x KS K-steps of 8, both operands K-major
  auto mma_stage = [&](int T, int KS, int NB, uint32_t a0, int a_sbo, uint32_t b0, int kb) {
    const uint32_t id = umma_idesc_tf32(NB, 0);
    for (int t = 0; t < T; ++t)
      for (int ks = 0; ks < KS; ++ks)
        umma_tf32(tcol + t * NB, umma_sdesc(a0 + t * 16 * a_sbo + ks * 256, 128, a_sbo),
                  umma_sdesc(b0 + ks * 256, 128, (kb / 4) * 128), id, ks > 0 ? 1u : 0u);
  };
  auto run = [&](int T, int KS, int NB, uint32_t a0, int a_sbo, uint32_t b0, int kb) {
    if (leader) {
      tc_fence_after();
      mma_stage(T, KS, NB, a0, a_sbo, b0, kb);
      umma_commit(mbar);
    }
    wait_mma();
  };

  int it = 0;
  const int first = blockIdx.x * U + u;
  if (leader && first < a.n_patches) issue(first, 0);
  for (int pp = first; pp < a.n_patches; pp += gstride, ++it) {
    const int sl = C::SLOTS == 2 ? (it & 1) : 0;
    unsigned char *work = slots + sl * C::SLOT;
    const float *bbox = reinterpret_cast<const float *>(work + C::WORK);
    const uint32_t wsa = smem_u32(work);
    if (C::SLOTS == 2 && leader && pp + gstride < a.n_patches) issue(pp + gstride, sl ^ 1);
    int fx, fy, fz;
    patch_xyz(pp, fx, fy, fz);
    const int xo = fx & 3;
    if (!mbar_wait_bounded(&tbar[sl], C::SLOTS == 2 ? (it >> 1) & 1 : it & 1)) {
      atomicExch(err, 1);
      s_abort[u] = 1;
    }
    float *const wf = reinterpret_cast<float *>(work);
    if (!a.zero_x) {
      // ring form: the interior of x does not enter the residual
      for (int e = ut; e < M * M * M; e += 128) {
        const int xl = 1 + e % M, y = 1 + (e / M) % M, z = 1 + e / (M * M), xx = xl + xo;
        wf[(((y >> 3) * N1 + z) * C::SBO1 + (xx >> 2) * 128 + ((y & 7) << 4) + ((xx & 3) << 2)) >> 2] = 0.f;
      }
    }
    stage_sync();
    if (s_abort[u]) break;  // uniform: read after the unit barrier

    float r[C::KF];  // residual of this thread's z-line (S3 epilogue)
    if (!a.zero_x) {
      // ---- S1: x ------------------------------------------------------------
      run(C::T1, C::KS1, C::NB1, wsa, C::SBO1, s_base + C::OFF_B1 + xo * C::SB1, C::K1);
      for (int t = 0; t < C::T1; ++t) {
        float v[C::NB1];
#pragma unroll
        for (int c = 0; c < C::NB1; c += 16) tmem_ld16(tme + t * C::NB1 + c, v + c);
        const int m = t * 128 + ut, g = m >> 3, z = g % N1, y = (m & 7) + 8 * (g / N1);
        if (g < C::YH * N1 && y < N1) {
#pragma unroll
          for (int xi = 0; xi < M; ++xi)
            *reinterpret_cast<float2 *>(work + km_off(xi + M * z, 2 * y, C::SBO2)) =
                make_float2(to_tf32(v[xi]), to_tf32(v[M + xi]));
        }
      }
      stage_sync();
      // ---- S2: y ------------------------------------------------------------
      run(C::T2, C::KS2, C::NB2, wsa, C::SBO2, s_base + C::OFF_B2, C::K2);
      for (int t = 0; t < C::T2; ++t) {
        float v[C::NB2];
#pragma unroll
        for (int c = 0; c < C::NB2; c += 16) tmem_ld16(tme + t * C::NB2 + c, v + c);
        const int m = t * 128 + ut, z = m / M, xi = m % M;
        if (z < N1) {
#pragma unroll
          for (int yi = 0; yi < M; ++yi)
            *reinterpret_cast<float2 *>(work + km_off(xi + M * yi, 2 * z, C::SBO3)) =
                make_float2(to_tf32(v[yi]), to_tf32(v[M + yi]));
        }
      }
      stage_sync();
      // ---- S3: z, -s A x ------------------------------------------------------
      run(C::T3, C::KS3, C::NB3, wsa, C::SBO3, s_base + C::OFF_B3, C::K3);
    }
    // residual r = b - s A x on this thread's z-line, written back on the same
    // row as the S^T_z operand (K = zi)
    for (int t = 0; t < C::TF; ++t) {
      float v[C::NB3];
      if (!a.zero_x) {
#pragma unroll
        for (int c = 0; c < C::NB3; c += 16) tmem_ld16(tme + t * C::NB3 + c, v + c);
      } else {
#pragma unroll
        for (int c = 0; c < C::NB3; ++c) v[c] = 0.f;
      }
      const int m = t * 128 + ut, yi = m / M, xi = m % M;
      if (yi < M) {
#pragma unroll
        for (int zi = 0; zi < C::KF; ++zi)
          r[zi] = zi < M ? to_tf32(bbox[(zi * M + yi) * C::XW + xo + 1 + xi] + v[zi]) : 0.f;
#pragma unroll
        for (int c = 0; c < C::KF / 4; ++c)
          *reinterpret_cast<float4 *>(work + km_off(m, 4 * c, C::SBOF)) =
              make_float4(r[4 * c], r[4 * c + 1], r[4 * c + 2], r[4 * c + 3]);
      }
    }
    stage_sync();
    // ---- S4..S9: fast-diagonalisation solve -------------------------------------
    // S4: S^T_z on rows (yi, xi) -> modes qz; rows become (qz, xi), K = yi
    run(C::TF, C::KSF, C::NBF, wsa, C::SBOF, s_base + C::OFF_BST, C::KF);
    for (int t = 0; t < C::TF; ++t) {
      float v[C::NBF];
#pragma unroll
      for (int c = 0; c < C::NBF; c += 16) tmem_ld16(tme + t * C::NBF + c, v + c);
      const int m = t * 128 + ut, yi = m / M, xi = m % M;
      if (yi < M) {
#pragma unroll
        for (int qz = 0; qz < M; ++qz) *reinterpret_cast<float *>(work + km_off(xi + M * qz, yi, C::SBOF)) = to_tf32(v[qz]);
      }
    }
    stage_sync();
    // S5: S^T_y on rows (qz, xi) -> qy; rows become (qz, qy), K = xi
    run(C::TF, C::KSF, C::NBF, wsa, C::SBOF, s_base + C::OFF_BST, C::KF);
    for (int t = 0; t < C::TF; ++t) {
      float v[C::NBF];
#pragma unroll
      for (int c = 0; c < C::NBF; c += 16) tmem_ld16(tme + t * C::NBF + c, v + c);
      const int m = t * 128 + ut, qz = m / M, xi = m % M;
      if (qz < M) {
#pragma unroll
        for (int qy = 0; qy < M; ++qy) *reinterpret_cast<float *>(work + km_off(qy + M * qz, xi, C::SBOF)) = to_tf32(v[qy]);
      }
    }
    stage_sync();
    // S6: S^T_x on rows (qz, qy) -> qx, eigenvalue scaling; same rows, K = qx
    run(C::TF, C::KSF, C::NBF, wsa, C::SBOF, s_base + C::OFF_BST, C::KF);
    for (int t = 0; t < C::TF; ++t) {
      float v[C::NBF];
#pragma unroll
      for (int c = 0; c < C::NBF; c += 16) tmem_ld16(tme + t * C::NBF + c, v + c);
      const int m = t * 128 + ut, qz = m / M, qy = m % M;
      if (qz < M) {
        float w[C::KF];
#pragma unroll
        for (int qx = 0; qx < C::KF; ++qx) w[qx] = qx < M ? to_tf32(v[qx] * RL[(qz * M + qy) * M + qx]) : 0.f;
#pragma unroll
        for (int c = 0; c < C::KF / 4; ++c)
          *reinterpret_cast<float4 *>(work + km_off(m, 4 * c, C::SBOF)) =
              make_float4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]);
      }
    }
    stage_sync();
    // S7: S_x on rows (qz, qy) -> x; rows become (qz, x), K = qy
    run(C::TF, C::KSF, C::NBF, wsa, C::SBOF, s_base + C::OFF_BS, C::KF);
    for (int t = 0; t < C::TF; ++t) {
      float v[C::NBF];
#pragma unroll
      for (int c = 0; c < C::NBF; c += 16) tmem_ld16(tme + t * C::NBF + c, v + c);
      const int m = t * 128 + ut, qz = m / M, qy = m % M;
      if (qz < M) {
#pragma unroll
        for (int xl = 0; xl < M; ++xl) *reinterpret_cast<float *>(work + km_off(xl + M * qz, qy, C::SBOF)) = to_tf32(v[xl]);
      }
    }
    stage_sync();
    // S8: S_y on rows (qz, x) -> y; rows become (y, x), K = qz
    run(C::TF, C::KSF, C::NBF, wsa, C::SBOF, s_base + C::OFF_BS, C::KF);
    for (int t = 0; t < C::TF; ++t) {
      float v[C::NBF];
#pragma unroll
      for (int c = 0; c < C::NBF; c += 16) tmem_ld16(tme + t * C::NBF + c, v + c);
      const int m = t * 128 + ut, qz = m / M, xl = m % M;
      if (qz < M) {
#pragma unroll
        for (int y = 0; y < M; ++y) *reinterpret_cast<float *>(work + km_off(xl + M * y, qz, C::SBOF)) = to_tf32(v[y]);
      }
    }
    stage_sync();
    // S9: S_z on rows (y, x) -> z, stored to x_I
    run(C::TF, C::KSF, C::NBF, wsa, C::SBOF, s_base + C::OFF_BS, C::KF);
    for (int t = 0; t < C::TF; ++t) {
      float v[C::NBF];
#pragma unroll
      for (int c = 0; c < C::NBF; c += 16) tmem_ld16(tme + t * C::NBF + c, v + c);
      const int m = t * 128 + ut, y = m / M, xl = m % M;
      if (y < M) {
        float *dst = x + (fx + 1 + xl) + (fy + 1 + y) * a.sy + (fz + 1) * a.sz;
#pragma unroll
        for (int z = 0; z < M; ++z) dst[z * a.sz] = v[z];
      }
    }
    // TMEM reads and shared-memory operand reads of this patch are complete
    // before the unit's next MMAs and TMA loads
    tc_fence_before();
    named_bar(1 + u, 128);
    // one slot: the next patch is fetched once this one has left the slot
    if (C::SLOTS == 1 && leader && pp + gstride < a.n_patches) {
      fence_proxy_async_smem();
      issue(pp + gstride, 0);
    }
  }
  // a unit that stopped early waits (bounded) for its prefetch still in flight
  // (with one slot no load is issued ahead of the patch being solved)
  if (C::SLOTS == 2 && leader && s_abort[u]) {
    const int pp = first + it * gstride;
    if (pp + gstride < a.n_patches) (void)mbar_wait_bounded(&tbar[(it & 1) ^ 1], ((it + 1) >> 1) & 1);
  }
  tc_fence_before();
  __syncthreads();
  if (tid < 32) {
    tc_fence_after();
    tmem_dealloc(tmem, C::TMEM_COLS);
  }
}

}  // namespace tps
