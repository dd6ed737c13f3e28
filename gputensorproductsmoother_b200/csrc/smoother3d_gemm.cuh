// 3D vertex-patch smoother as one tensor-core GEMM over the patches of a
// colour (sm_100a, tcgen05 kind::tf32, FP32 accumulation in tensor memory).
//
// With a constant coefficient every patch has the same local problem, so the
// patch step of smoother3d_kernel (the reference's FUSED_CF kernel,
// include/loop_kernel.cuh:962-1060 with include/evaluate_kernel.cuh:501-590,
// 1327-1434, 2058-2163) in its ring form
//     x_I <- omega A_II^{-1} (b_I - A_IB x_B)
// is one fixed matrix G = [A_II^{-1} | -A_II^{-1} A_IB] (interior rows x box
// columns, reference-cell units) applied to the box vector u of the patch
// (u = b on the interior, s * x on the ring, s the level's stiffness scale),
// followed by the factor omega / s.  G commutes with the reflection of the box
// in z, so in the z-parity basis it splits into two blocks:
//     e_p = u(p) + u(N1-1-p), o_p = u(p) - u(N1-1-p)   (box planes, p < K; e_K = u(K))
//     E = G_E e, O = G_O o;  x(zi) = E_zi + O_zi, x(M-1-zi) = E_zi - O_zi, x(K-1) = E_K-1
// (the factors 1/2 of the basis change are folded into G_E and G_O, built in
// FP64 on the host by patch_gemm_image and rounded to TF32 once).
//
// One CTA per SM, persistent over tiles of 128 consecutive patches of the
// colour (the MMA rows).  Both GEMMs run chunk by chunk over K (CK entries per
// chunk) through a ring of shared-memory stages:
//   producer warps  gather e and o of their rows from global memory (the box
//                   planes z = p and N1-1-p, b or x), round to TF32 and store
//                   them in the K-major operand layout (one 128-byte core
//                   matrix per warp instruction: 8 patches x 4 K entries);
//   loader thread   copies the chunk's slices of G_E and G_O (pre-arranged in
//                   the operand layout) with cp.async.bulk, no tensor map;
//   MMA thread      issues the chunk's MMAs (M = 128 patches, N = the
//                   block's outputs, K = 8) and commits the stage back;
//   epilogue warps  (TMEM lanes = patches) read E and O, unfold, scale and
//                   store x_I.
// A tile's accumulators occupy NBE + NBO TMEM columns, so the next tile's
// MMAs wait for the epilogue; the producers and the loader run ahead through
// the stage ring meanwhile.  Every wait is bounded: a wait that runs out sets
// *err and the CTA's abort flag, every role then leaves its loop, the loader
// waits (bounded) for its copies still in flight, and TMEM is released.
#pragma once

#include <cuda.h>

#include "ptx.cuh"
#include "smoother3d.cuh"
#include "smoother3d_warp.cuh"
#include "tps_common.cuh"

namespace tps {

template <int K>
struct Pg3 {
  static constexpr int N1 = 2 * K + 1, M = 2 * K - 1;
  static constexpr int PL = N1 * N1, IPL = M * M;  // entries of a box plane, of an interior plane
  static constexpr int KE = (K + 1) * PL, KO = K * PL;
  static constexpr int NE = K * IPL, NO = (K - 1) * IPL;
  static constexpr int CK = 32;  // K entries per chunk: four MMA K-steps of 8
  static constexpr int CE = (KE + CK - 1) / CK, CO = (KO + CK - 1) / CK;
  static constexpr int NBE = (NE + 15) / 16 * 16, NBO = (NO + 15) / 16 * 16;
  static constexpr int SBO = (CK / 4) * 128;  // bytes between 8-row groups (K-major, no swizzle)
  static constexpr int A_BYTES = 16 * SBO;    // 128 rows of one block's chunk
  static constexpr int BE_BYTES = NBE / 8 * SBO, BO_BYTES = NBO / 8 * SBO;
  static constexpr int STAGE = 2 * A_BYTES + BE_BYTES + BO_BYTES;
  static constexpr int IMG_E = CE * BE_BYTES, IMG_O = CO * BO_BYTES;
  static constexpr int IMG_FLOATS = (IMG_E + IMG_O) / 4;
  static constexpr int KT = CE * CK;  // entries of the per-launch K table
  // producer warps in two teams that fill alternate chunks, so the global
  // loads of one chunk overlap the other team's
  static constexpr int TEAMS = 2, TEAM_WARPS = 4, PRODUCERS = TEAMS * TEAM_WARPS;
  static constexpr int ROWS_PER_PRODUCER = 128 / TEAM_WARPS;  // 8 quads of 4 rows
  static constexpr int NWARPS = 4 + PRODUCERS + 2;  // epilogue, producers, MMA, loader
  static constexpr int NT = 32 * NWARPS;
  static constexpr int W_MMA = 4 + PRODUCERS, W_LOAD = W_MMA + 1;
  // stages: as many as fit next to the K table and the barriers, a multiple of TEAMS
  static constexpr int FIXED = KT * 16 + 1024;
  static constexpr int STAGES_FIT = (232448 - FIXED - 1024) / STAGE;
  static constexpr int STAGES = (STAGES_FIT > 6 ? 6 : STAGES_FIT) / TEAMS * TEAMS;
  static constexpr int OFF_KT = STAGES * STAGE;
  static constexpr int OFF_BAR = OFF_KT + KT * 16;  // afull, bfull, empty per stage; acc_full, acc_empty, fin
  static constexpr int NBAR = 3 * STAGES + 3;
  static constexpr int OFF_MISC = OFF_BAR + 8 * NBAR;  // TMEM base, abort flag
  static constexpr int BYTES = OFF_MISC + 16;
  // tensor memory: E at column 0, O at NBE; the epilogue reads, for every
  // output row, 32-column windows at the row's 16-aligned start in both blocks
  static constexpr int LAST_WIN = ((NE - M) & ~15) + 32;
  static constexpr int COLS_USED = NBE + (LAST_WIN > NBO ? LAST_WIN : NBO);
  static constexpr int TMEM_COLS = COLS_USED <= 32 ? 32 : COLS_USED <= 64 ? 64 : COLS_USED <= 128 ? 128
                                 : COLS_USED <= 256 ? 256 : 512;
  static_assert(K >= 2 && K <= 4, "patch-GEMM smoother: degrees 2..4");
  static_assert(NBE <= 256 && NBO <= 256 && COLS_USED <= 512, "one MMA per block and chunk, accumulators in TMEM");
  static_assert(STAGES >= TEAMS && BYTES <= 232448, "shared memory");
  static_assert(BE_BYTES % 16 == 0 && BO_BYTES % 16 == 0 && STAGE % 128 == 0, "bulk copy sizes and alignment");
};

template <int K>
constexpr bool pg3_enabled()
{
  return K >= 2 && K <= 4;
}

// the B operand image of degree K (G_E chunks, then G_O chunks), written by
// the per-degree upload
template <int K>
__device__ __align__(128) float g_pg3_image[Pg3<K>::IMG_FLOATS];  // bulk-copy sources: 16-byte aligned

// one interior row of a patch (M = 2K-1 entries from box x = 1).  For K = 4
// the box origin is a multiple of 4 entries and so are the row pitches, so
// the row is 3 single entries and one 16-byte aligned vector.
template <int K>
__device__ __forceinline__ void store_row(float *d, const float *r)
{
  if constexpr (K == 4) {
    d[0] = r[0];
    d[1] = r[1];
    d[2] = r[2];
    *reinterpret_cast<float4 *>(d + 3) = make_float4(r[3], r[4], r[5], r[6]);
  } else {
#pragma unroll
    for (int xi = 0; xi < 2 * K - 1; ++xi) d[xi] = r[xi];
  }
}

template <int K>
__global__ void __launch_bounds__(Pg3<K>::NT, 1)
    smoother3d_gemm_kernel(float *__restrict__ x, const float *__restrict__ b, const Sm3Args a, float sc,
                           float fd, int *__restrict__ err)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  using C = Pg3<K>;
  constexpr int N1 = C::N1, M = C::M, PL = C::PL, IPL = C::IPL, CK = C::CK, ST = C::STAGES;
  extern __shared__ __align__(1024) unsigned char smem[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int4 *ktab = reinterpret_cast<int4 *>(smem + C::OFF_KT);
  uint64_t *afull = reinterpret_cast<uint64_t *>(smem + C::OFF_BAR);
  uint64_t *bfull = afull + ST, *empty = bfull + ST, *acc_full = empty + ST, *acc_empty = acc_full + 1;
  uint64_t *fin = acc_empty + 1;
  uint32_t *s_tmem = reinterpret_cast<uint32_t *>(smem + C::OFF_MISC);
  volatile int *s_abort = reinterpret_cast<volatile int *>(smem + C::OFF_MISC + 4);
  const int n_tiles = (a.n_patches + 127) / 128;

  // ---- set-up: K table, barriers, tensor memory --------------------------------
  // entry k: {offset of box plane p, of plane N1-1-p (-1: centre plane), 1 if the
  // entries come from b (patch interior), valid}; offsets from the box origin
  for (int k = tid; k < C::KT; k += C::NT) {
    int4 e = make_int4(0, -1, 0, 0);
    if (k < C::KE) {
      const int p = k / PL, s = k % PL, y = s / N1, xx = s % N1;
      const bool in_yx = y >= 1 && y <= N1 - 2 && xx >= 1 && xx <= N1 - 2;
      const int64_t o1 = p * a.sz + y * a.sy + xx, o2 = (N1 - 1 - p) * a.sz + y * a.sy + xx;
      e.x = static_cast<int>(o1);
      e.y = p < K ? static_cast<int>(o2) : -1;
      e.z = (p >= 1 && in_yx) ? 1 : 0;  // planes 1..N1-2 and an interior (y, x)
      e.w = 1;
    }
    ktab[k] = e;
  }
  if (tid == 0) {
    for (int s = 0; s < ST; ++s) {
      mbar_init(&afull[s], C::TEAM_WARPS);
      mbar_init(&bfull[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(acc_full, 1);
    mbar_init(acc_empty, 4);
    mbar_init(fin, 1);
    *s_abort = 0;
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(s_tmem, C::TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  const uint32_t s_base = smem_u32(smem);
  auto fail = [&]() {
    atomicExch(err, 1);
    *s_abort = 1;
  };

  if (warp >= 4 && warp < C::W_MMA) {
    // ---- producers: team tm fills the chunks gc with gc % TEAMS == tm.  A warp
    // instruction covers 4 rows (lane / 8) x 8 consecutive K entries (lane % 8):
    // 32-byte runs of 4 neighbouring patches in global memory, 2-way bank
    // conflicts in the operand stores.  Warp pw of the team owns rows
    // 32 pw .. 32 pw + 31.  All global loads of a chunk are issued,
    // unconditionally and in bounds, before the stage is awaited.
    constexpr int NI = C::ROWS_PER_PRODUCER / 4, NQ = CK / 8;
    const int tm = (warp - 4) / C::TEAM_WARPS, pw = (warp - 4) % C::TEAM_WARPS, rp = lane >> 3, kk = lane & 7;
    int gc = 0;
    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
      // box origins as 32-bit offsets (a level holds fewer than 2^31 entries)
      int orig[NI];
      unsigned valid = 0;
#pragma unroll
      for (int i = 0; i < NI; ++i) {
        const int j = tile * 128 + C::ROWS_PER_PRODUCER * pw + 4 * i + rp;
        int fx = 0, fy = 0, fz = 0;
        if (j < a.n_patches) {
          valid |= 1u << i;
          wp_patch_xyz(a, j, K, fx, fy, fz);
        }
        // a row past the colour reads the box at 0 (in bounds)
        orig[i] = static_cast<int>(fx + fy * a.sy + fz * a.sz);
      }
      for (int c = 0; c < C::CE; ++c, ++gc) {
        if (gc % C::TEAMS != tm) continue;
        const int s = gc % ST, round = gc / ST;
        float u1[NI][NQ], u2[NI][NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
          const int4 t = ktab[c * CK + 8 * q + kk];
          const float *src = t.z ? b : x;
#pragma unroll
          for (int i = 0; i < NI; ++i) {
            u1[i][q] = src[static_cast<unsigned>(orig[i] + t.x)];
            u2[i][q] = src[static_cast<unsigned>(orig[i] + (t.y >= 0 ? t.y : t.x))];
          }
        }
        if (round > 0 && !mbar_wait_bounded(&empty[s], (round - 1) & 1)) fail();
        if (*s_abort) break;
        unsigned char *ae = smem + s * C::STAGE, *ao = ae + C::A_BYTES;
        const bool odd = c < C::CO;
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
          const int4 t = ktab[c * CK + 8 * q + kk];
          const float f = t.z ? 1.f : sc;
          const bool use = t.w && (t.z || !a.zero_x);
          const bool pair = t.y >= 0;
          const int kc = 8 * q + kk;  // K entry within the chunk
#pragma unroll
          for (int i = 0; i < NI; ++i) {
            const bool keep = use && ((valid >> i) & 1u);
            const float v1 = keep ? u1[i][q] : 0.f, v2 = (keep && pair) ? u2[i][q] : 0.f;
            const int m = C::ROWS_PER_PRODUCER * pw + 4 * i + rp;
            const int off = (m >> 3) * C::SBO + (m & 7) * 16 + (kc >> 2) * 128 + (kc & 3) * 4;
            *reinterpret_cast<float *>(ae + off) = to_tf32(f * (v1 + v2));
            if (odd) *reinterpret_cast<float *>(ao + off) = to_tf32(f * (v1 - v2));
          }
        }
        fence_proxy_async_smem();  // the operand stores are read by the tensor cores
        __syncwarp();
        if (lane == 0) mbar_arrive(&afull[s]);
      }
      if (*s_abort) break;
    }
  } else if (warp == C::W_LOAD) {
    // ---- loader: the chunk's slices of G_E and G_O --------------------------------
    if (lane == 0) {
      const float *img = g_pg3_image<K>;
      const unsigned char *ge = reinterpret_cast<const unsigned char *>(img);
      const unsigned char *go = ge + C::IMG_E;
      int gc = 0;
      for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        for (int c = 0; c < C::CE; ++c, ++gc) {
          const int s = gc % ST, round = gc / ST;
          if (round > 0 && !mbar_wait_bounded(&empty[s], (round - 1) & 1)) fail();
          if (*s_abort) break;
          unsigned char *be = smem + s * C::STAGE + 2 * C::A_BYTES, *bo = be + C::BE_BYTES;
          const bool odd = c < C::CO;
          mbar_arrive_expect_tx(&bfull[s], C::BE_BYTES + (odd ? C::BO_BYTES : 0));
          bulk_load(be, ge + c * C::BE_BYTES, C::BE_BYTES, &bfull[s]);
          if (odd) bulk_load(bo, go + c * C::BO_BYTES, C::BO_BYTES, &bfull[s]);
        }
        if (*s_abort) break;
      }
      // copies still in flight when the CTA gave up: wait for them (bounded)
      if (*s_abort) {
        const int first = gc > ST ? gc - ST : 0;
        for (int g = first; g < gc; ++g) (void)mbar_wait_bounded(&bfull[g % ST], (g / ST) & 1);
      }
    }
  } else if (warp == C::W_MMA) {
    // ---- MMA issue ------------------------------------------------------------------
    if (lane == 0) {
      const uint32_t ide = umma_idesc_tf32(C::NBE, 0), ido = umma_idesc_tf32(C::NBO, 0);
      int gc = 0, ti = 0;
      for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, ++ti) {
        if (ti > 0 && !mbar_wait_bounded(acc_empty, (ti - 1) & 1)) fail();
        if (*s_abort) break;
        tc_fence_after();
        for (int c = 0; c < C::CE; ++c, ++gc) {
          const int s = gc % ST, ph = (gc / ST) & 1;
          if (!mbar_wait_bounded(&afull[s], ph) || !mbar_wait_bounded(&bfull[s], ph)) fail();
          if (*s_abort) break;
          tc_fence_after();
          const uint32_t ae = s_base + s * C::STAGE, ao = ae + C::A_BYTES;
          const uint32_t be = ae + 2 * C::A_BYTES, bo = be + C::BE_BYTES;
#pragma unroll
          for (int ks = 0; ks < CK / 8; ++ks) {
            const uint32_t acc = (c > 0 || ks > 0) ? 1u : 0u;
            umma_tf32(tmem, umma_sdesc(ae + ks * 256, 128, C::SBO), umma_sdesc(be + ks * 256, 128, C::SBO), ide,
                      acc);
            if (c < C::CO)
              umma_tf32(tmem + C::NBE, umma_sdesc(ao + ks * 256, 128, C::SBO),
                        umma_sdesc(bo + ks * 256, 128, C::SBO), ido, acc);
          }
          umma_commit(&empty[s]);  // the stage is free once these MMAs have read it
        }
        if (*s_abort) break;
        umma_commit(acc_full);
      }
      // every MMA issued here has completed before tensor memory is released
      umma_commit(fin);
      if (!mbar_wait_bounded(fin, 0)) fail();
    }
  } else {
    // ---- epilogue: TMEM lane = row = patch ----------------------------------------
    const int m = tid;  // warps 0..3
    const uint32_t trow = tmem + (static_cast<uint32_t>(32 * warp) << 16);
    int ti = 0;
    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, ++ti) {
      if (!mbar_wait_bounded(acc_full, ti & 1)) fail();
      if (*s_abort) break;
      tc_fence_after();
      const int j = tile * 128 + m;
      const bool valid = j < a.n_patches;
      int fx = 0, fy = 0, fz = 0;
      if (valid) wp_patch_xyz(a, j, K, fx, fy, fz);
      float *const xp = x + (fx + 1 + (fy + 1) * a.sy + (fz + 1) * a.sz);
      const int sy32 = static_cast<int>(a.sy), sz32 = static_cast<int>(a.sz);
#pragma unroll
      for (int zp = 0; zp < K; ++zp) {
#pragma unroll
        for (int yi = 0; yi < M; ++yi) {
          // the row's M columns of E and of O lie in 32-column windows at 16-aligned starts
          const int c0 = zp * IPL + yi * M, b0 = c0 & ~15;
          float v[64];  // E window, then O window
          tmem_ld16x4(trow + b0, trow + b0 + 16, trow + C::NBE + b0, trow + C::NBE + b0 + 16, v);
          if (valid) {
            float r1[M], r2[M];
#pragma unroll
            for (int xi = 0; xi < M; ++xi) {
              const float e = v[c0 - b0 + xi], o = zp < K - 1 ? v[32 + c0 - b0 + xi] : 0.f;
              r1[xi] = fd * (e + o);
              r2[xi] = fd * (e - o);
            }
            store_row<K>(xp + zp * sz32 + yi * sy32, r1);
            if (zp < K - 1) store_row<K>(xp + (M - 1 - zp) * sz32 + yi * sy32, r2);
          }
        }
      }
      tc_fence_before();  // the TMEM reads precede the next tile's MMAs
      __syncwarp();
      if (lane == 0) mbar_arrive(acc_empty);
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, C::TMEM_COLS);
  }
}

}  // namespace tps
