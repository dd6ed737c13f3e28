// 3D vertex-patch smoother as one tensor-core GEMM over the patches of a
// colour, degree 4, with one producer thread per patch (sm_100a, tcgen05
// kind::tf32, FP32 accumulation in tensor memory).
//
// Algebra as smoother3d_gemm_kernel (the reference's FUSED_CF patch step,
// include/loop_kernel.cuh:962-1060 with include/evaluate_kernel.cuh:501-590,
// 1327-1434, 2058-2163, in the ring form x_I <- omega A_II^{-1}(b_I - A_IB x_B)):
// one fixed matrix G = [A_II^{-1} | -A_II^{-1} A_IB] applied to the box
// vector u of every patch (b inside, s * x on the ring), split by the
// z-reflection into the blocks G_E and G_O, then the factor omega / s.
//
// What is different: the operand producer.  The earlier kernel gathered 4
// patches x 8 K entries per warp instruction from global memory (11 sectors
// per request, L1-bound).  Here the K columns are ordered so that a chunk is
// RPC box rows (x = 0..7) of one plane pair (three rows, 24 columns, with one
// TF32 pass; one row with three passes), the x = 8 entries coming last
// (patch_gemm_image_ordered, order 1).  At degree 4 a
// patch's box origin is a multiple of 4 entries and so are the padded row
// pitches, so a producer thread -- one per patch, i.e. per MMA row -- reads
// each box row of its patch as two 16-byte vectors (ring rows from x, the
// interior rows' entries 1..7 from b), folds the plane pair (e = u(p) +
// u(8-p), o = u(p) - u(8-p)), rounds to TF32 and writes each group of 4 K
// entries with one 16-byte store: the 8 lanes of a quarter warp fill one
// 128-byte core-matrix row group, so the operand stores are free of bank
// conflicts.
//
// With PASSES = 3 the products are formed as a_hi b_hi + a_hi b_lo + a_lo b_hi
// with a_lo = tf32(a - a_hi) and b_lo from the split G image (three TF32 MMAs
// per K step and block): about FP32 accuracy per product, FP32 accumulation.
//
// Roles (persistent, one CTA per SM, tiles of 128 consecutive patches of the
// colour): warps 0-3 epilogue (TMEM lane = patch), then TEAMS teams of 4
// producer warps that fill chunks in turn (thread = patch; three teams with
// one TF32 pass, four with three), one warp that issues the MMAs and one
// that copies G chunks with cp.async.bulk (this GPU's memory into this CTA
// only).  Every wait is
// bounded; a wait that runs out sets *err and the CTA's abort flag, every role
// leaves its loop, the loader waits (bounded) for its copies in flight, and
// TMEM is released.
#pragma once

#include <cuda.h>

#include "ptx.cuh"
#include "smoother3d.cuh"
#include "smoother3d_gemm.cuh"
#include "smoother3d_warp.cuh"
#include "tps_common.cuh"

namespace tps {

template <int K, int PASSES>
struct Pgv {
  static_assert(K == 4, "vector producers need box rows aligned to 16 bytes: degree 4");
  static_assert(PASSES == 1 || PASSES == 3, "TF32 (1) or three-product TF32 (3)");
  static constexpr int N1 = 2 * K + 1, M = 2 * K - 1, PL = N1 * N1, IPL = M * M;
  static constexpr int RW = N1 - 1;                     // vector part of a box row
  static constexpr int RPP = N1 * RW;                   // row entries of one plane pair
  static constexpr int KE = (K + 1) * PL, KO = K * PL;  // real columns of G_E, G_O
  // box rows per chunk: three (24 columns, 3 MMA K steps) with one TF32
  // pass; one with three passes, whose stages hold two precision parts
  static constexpr int RPC = PASSES == 1 ? 3 : 1;
  static constexpr int CPP = N1 / RPC;                  // row chunks per plane pair
  static constexpr int CK = RPC * RW;
  static constexpr int CE = (KE + CK - 1) / CK, CO = (KO + CK - 1) / CK;
  static constexpr int CE_ROWS = (K + 1) * CPP, CO_ROWS = K * CPP;  // row chunks
  static constexpr int NE = K * IPL, NO = (K - 1) * IPL;
  static constexpr int NBE = (NE + 15) / 16 * 16, NBO = (NO + 15) / 16 * 16;
  static constexpr int SBO = (CK / 4) * 128;  // bytes between 8-row groups (K-major, no swizzle)
  static constexpr int A_BYTES = 16 * SBO;    // 128 rows of one block's chunk (one precision part)
  static constexpr int BE_BYTES = NBE / 8 * SBO, BO_BYTES = NBO / 8 * SBO;
  static constexpr int PARTS = PASSES == 1 ? 1 : 2;  // hi (and lo) parts of A and of B
  static constexpr int STAGE = PARTS * (2 * A_BYTES + BE_BYTES + BO_BYTES);
  static constexpr int IMG_E = CE * BE_BYTES, IMG_O = CO * BO_BYTES;
  static constexpr int IMG_FLOATS = PARTS * (IMG_E + IMG_O) / 4;
  static constexpr int STAGES_FIT = (232448 - 2048) / STAGE;
  static constexpr int STAGES = STAGES_FIT > 6 ? 6 : STAGES_FIT;
  // warps: 0-3 epilogue, TEAMS producer teams of 4 (team t fills the chunks
  // gc with gc % TEAMS == t, so the teams' global loads are in flight
  // together), MMA issue, loader.  A team waits on a stage's "empty" barrier
  // for the consumption of the chunk ST chunks back; its previous wait
  // guaranteed the chunks up to TEAMS + ST back, so with TEAMS <= ST the
  // barrier is never two phases behind the awaited one (the parity test of
  // an mbarrier cannot tell a phase from the one two later)
  static constexpr int TEAMS = STAGES < 4 ? STAGES : 4;
  static constexpr int NWARPS = 4 + 4 * TEAMS + 2, NT = 32 * NWARPS;
  static constexpr int W_PROD = 4, W_MMA = 4 + 4 * TEAMS, W_LOAD = W_MMA + 1;
  static constexpr int OFF_BAR = STAGES * STAGE;
  static constexpr int NBAR = 3 * STAGES + 3;  // afull, bfull, empty per stage; acc_full, acc_empty, fin
  static constexpr int OFF_MISC = OFF_BAR + 8 * NBAR;
  static constexpr int BYTES = OFF_MISC + 16;
  static constexpr int LAST_WIN = ((NE - M) & ~15) + 32;
  static constexpr int COLS_USED = NBE + (LAST_WIN > NBO ? LAST_WIN : NBO);
  static constexpr int TMEM_COLS = 512;
  static_assert(STAGES >= 2 && BYTES <= 232448, "shared memory");
  static_assert(TEAMS <= STAGES, "stage barrier parity: a team stays within one phase");
  static_assert(COLS_USED <= TMEM_COLS && NBE <= 256 && NBO <= 256, "accumulators in TMEM, one MMA per block");
  static_assert(STAGE % 128 == 0 && BE_BYTES % 16 == 0 && BO_BYTES % 16 == 0, "alignment");
  static_assert(CPP * RPC == N1 && CE_ROWS * CK == (K + 1) * RPP && CO_ROWS * CK == K * RPP, "row chunks");
};

// B operand images of degree 4 (order 1): TF32, and hi/lo for three passes
template <int K, int PASSES>
__device__ __align__(128) float g_pgv_image[Pgv<K, PASSES>::IMG_FLOATS];  // bulk-copy sources: 16-byte aligned

// split a value into its TF32 part and the TF32 residual
__device__ __forceinline__ void tf32_split(float v, float &hi, float &lo)
{
  hi = to_tf32(v);
  lo = to_tf32(v - hi);
}

template <int K, int PASSES>
__global__ void __launch_bounds__(Pgv<K, PASSES>::NT, 1)
    smoother3d_pgemm_kernel(float *__restrict__ x, const float *__restrict__ b, const Sm3Args a, float sc,
                            float fd, int *__restrict__ err)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  using C = Pgv<K, PASSES>;
  constexpr int N1 = C::N1, M = C::M, IPL = C::IPL, CK = C::CK, ST = C::STAGES, RW = C::RW, RPC = C::RPC;
  extern __shared__ __align__(1024) unsigned char smem[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint64_t *afull = reinterpret_cast<uint64_t *>(smem + C::OFF_BAR);
  uint64_t *bfull = afull + ST, *empty = bfull + ST, *acc_full = empty + ST, *acc_empty = acc_full + 1;
  uint64_t *fin = acc_empty + 1;
  uint32_t *s_tmem = reinterpret_cast<uint32_t *>(smem + C::OFF_MISC);
  volatile int *s_abort = reinterpret_cast<volatile int *>(smem + C::OFF_MISC + 4);
  const int n_tiles = (a.n_patches + 127) / 128;

  if (tid == 0) {
    for (int s = 0; s < ST; ++s) {
      mbar_init(&afull[s], 4);  // one arrival per producer warp
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

  if (warp >= C::W_PROD && warp < C::W_MMA) {
    // ---- producers: thread = patch (row m of the tile) ----------------------------
    const int team = (warp - C::W_PROD) / 4;
    const int m = tid - 32 * (C::W_PROD + 4 * team);
    const int sy = static_cast<int>(a.sy), sz = static_cast<int>(a.sz);
    // operand offset of row m, entries 4q..4q+3 of a chunk at + q * 128
    const int arow = (m >> 3) * C::SBO + (m & 7) * 16;
    int gc = 0;
    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
      const int j = tile * 128 + m;
      const bool valid = j < a.n_patches;
      int fx = 0, fy = 0, fz = 0;
      if (valid) wp_patch_xyz(a, j, K, fx, fy, fz);
      const int org = fx + fy * sy + fz * sz;  // box origin (a level holds < 2^31 entries)
      const bool use_x = !a.zero_x;
      for (int c = 0; c < C::CE; ++c, ++gc) {
        if (gc % C::TEAMS != team) continue;
        const int s = gc % ST, round = gc / ST;
        // values of this chunk: E (and O) entries 0..CK-1, hi (and lo) parts
        float ev[CK], ov[CK];
        const bool has_o = c < C::CO;
        if (c < C::CE_ROWS) {
          // RPC box rows y0.. (x = 0..7) of plane pair p
          const int p = c / C::CPP, y0 = (c % C::CPP) * RPC;
          const bool zin = p >= 1;  // planes p and 8-p are interior planes (p <= K)
#pragma unroll
          for (int r = 0; r < RPC; ++r) {
            const int y = y0 + r;
            const bool inner = zin && y >= 1 && y <= N1 - 2;
            float up[RW], uq[RW];
#pragma unroll
            for (int q = 0; q < RW; ++q) up[q] = uq[q] = 0.f;
            if (valid) {
              const int rp = org + y * sy + p * sz, rq = org + y * sy + (N1 - 1 - p) * sz;
              const bool pair = p < K;  // the centre plane pair is one plane
              if (inner) {
                // entry 0 (ring) from x, entries 1..7 (interior) from b
                const float4 b0 = __ldg(reinterpret_cast<const float4 *>(b + rp));
                const float4 b1 = __ldg(reinterpret_cast<const float4 *>(b + rp) + 1);
                up[0] = use_x ? sc * x[rp] : 0.f;
                up[1] = b0.y; up[2] = b0.z; up[3] = b0.w; up[4] = b1.x; up[5] = b1.y; up[6] = b1.z; up[7] = b1.w;
                if (pair) {
                  const float4 c0 = __ldg(reinterpret_cast<const float4 *>(b + rq));
                  const float4 c1 = __ldg(reinterpret_cast<const float4 *>(b + rq) + 1);
                  uq[0] = use_x ? sc * x[rq] : 0.f;
                  uq[1] = c0.y; uq[2] = c0.z; uq[3] = c0.w; uq[4] = c1.x; uq[5] = c1.y; uq[6] = c1.z; uq[7] = c1.w;
                }
              } else if (use_x) {
                const float4 x0 = *reinterpret_cast<const float4 *>(x + rp);
                const float4 x1 = *(reinterpret_cast<const float4 *>(x + rp) + 1);
                up[0] = sc * x0.x; up[1] = sc * x0.y; up[2] = sc * x0.z; up[3] = sc * x0.w;
                up[4] = sc * x1.x; up[5] = sc * x1.y; up[6] = sc * x1.z; up[7] = sc * x1.w;
                if (pair) {
                  const float4 y0v = *reinterpret_cast<const float4 *>(x + rq);
                  const float4 y1v = *(reinterpret_cast<const float4 *>(x + rq) + 1);
                  uq[0] = sc * y0v.x; uq[1] = sc * y0v.y; uq[2] = sc * y0v.z; uq[3] = sc * y0v.w;
                  uq[4] = sc * y1v.x; uq[5] = sc * y1v.y; uq[6] = sc * y1v.z; uq[7] = sc * y1v.w;
                }
              }
            }
#pragma unroll
            for (int q = 0; q < RW; ++q) {
              // the centre plane pair (p = K) is a single plane: e = u(K)
              ev[r * RW + q] = p == K ? up[q] : up[q] + uq[q];
              ov[r * RW + q] = up[q] - uq[q];
            }
          }
        } else {
          // x = 8 entries: E columns (c - CE_ROWS) * CK + kk -> (plane pair, y);
          // the O block's own x = 8 chunks start at CO_ROWS
#pragma unroll
          for (int kk = 0; kk < CK; ++kk) {
            float e = 0.f, o = 0.f;
            const int ce_col = (c - C::CE_ROWS) * CK + kk;  // E: index into (K+1) * N1 entries
            if (valid && use_x && ce_col < (K + 1) * N1) {
              const int p = ce_col / N1, y = ce_col % N1;
              const float u1 = x[org + RW + y * sy + p * sz];
              const float u2 = p == K ? 0.f : x[org + RW + y * sy + (N1 - 1 - p) * sz];
              e = sc * (u1 + u2);
            }
            ev[kk] = e;
            ov[kk] = o;
          }
        }
        if (has_o && c >= C::CO_ROWS) {
#pragma unroll
          for (int kk = 0; kk < CK; ++kk) {
            float o = 0.f;
            const int co_col = (c - C::CO_ROWS) * CK + kk;  // O: index into K * N1 entries
            if (valid && use_x && co_col < K * N1) {
              const int p = co_col / N1, y = co_col % N1;
              o = sc * (x[org + RW + y * sy + p * sz] - x[org + RW + y * sy + (N1 - 1 - p) * sz]);
            }
            ov[kk] = o;
          }
        }
        if (round > 0 && !mbar_wait_bounded(&empty[s], (round - 1) & 1)) fail();
        if (*s_abort) break;
        unsigned char *st = smem + s * C::STAGE;
        // parts of the stage: [A_E hi][A_O hi]([A_E lo][A_O lo]) [B ...]
#pragma unroll
        for (int q = 0; q < CK / 4; ++q) {
          float4 eh, el, oh, ol;
          tf32_split(ev[4 * q], eh.x, el.x);
          tf32_split(ev[4 * q + 1], eh.y, el.y);
          tf32_split(ev[4 * q + 2], eh.z, el.z);
          tf32_split(ev[4 * q + 3], eh.w, el.w);
          *reinterpret_cast<float4 *>(st + arow + q * 128) = eh;
          if constexpr (PASSES == 3) *reinterpret_cast<float4 *>(st + 2 * C::A_BYTES + arow + q * 128) = el;
          if (has_o) {
            tf32_split(ov[4 * q], oh.x, ol.x);
            tf32_split(ov[4 * q + 1], oh.y, ol.y);
            tf32_split(ov[4 * q + 2], oh.z, ol.z);
            tf32_split(ov[4 * q + 3], oh.w, ol.w);
            *reinterpret_cast<float4 *>(st + C::A_BYTES + arow + q * 128) = oh;
            if constexpr (PASSES == 3) *reinterpret_cast<float4 *>(st + 3 * C::A_BYTES + arow + q * 128) = ol;
          }
        }
        fence_proxy_async_smem();  // the operand stores are read by the tensor cores
        __syncwarp();
        if (lane == 0) mbar_arrive(&afull[s]);
      }
      if (*s_abort) break;
    }
  } else if (warp == C::W_LOAD) {
    // ---- loader: the chunk's slices of G_E and G_O (hi, and lo for 3 passes) ----
    if (lane == 0) {
      const unsigned char *img = reinterpret_cast<const unsigned char *>(g_pgv_image<K, PASSES>);
      constexpr int ONE = C::IMG_E + C::IMG_O;  // bytes of one precision part of the image
      int gc = 0;
      for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        for (int c = 0; c < C::CE; ++c, ++gc) {
          const int s = gc % ST, round = gc / ST;
          if (round > 0 && !mbar_wait_bounded(&empty[s], (round - 1) & 1)) fail();
          if (*s_abort) break;
          unsigned char *bb = smem + s * C::STAGE + C::PARTS * 2 * C::A_BYTES;
          const bool odd = c < C::CO;
          const uint32_t per_part = C::BE_BYTES + (odd ? C::BO_BYTES : 0);
          mbar_arrive_expect_tx(&bfull[s], C::PARTS * per_part);
#pragma unroll
          for (int part = 0; part < C::PARTS; ++part) {
            unsigned char *be = bb + part * (C::BE_BYTES + C::BO_BYTES), *bo = be + C::BE_BYTES;
            bulk_load(be, img + part * ONE + c * C::BE_BYTES, C::BE_BYTES, &bfull[s]);
            if (odd) bulk_load(bo, img + part * ONE + C::IMG_E + c * C::BO_BYTES, C::BO_BYTES, &bfull[s]);
          }
        }
        if (*s_abort) break;
      }
      if (*s_abort) {
        const int first = gc > ST ? gc - ST : 0;
        for (int g = first; g < gc; ++g) (void)mbar_wait_bounded(&bfull[g % ST], (g / ST) & 1);
      }
    }
  } else if (warp == C::W_MMA) {
    // ---- MMA issue --------------------------------------------------------------
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
          const uint32_t st = s_base + s * C::STAGE;
          const uint32_t ae_hi = st, ao_hi = st + C::A_BYTES;
          const uint32_t ae_lo = st + 2 * C::A_BYTES, ao_lo = ae_lo + C::A_BYTES;
          const uint32_t bb = st + C::PARTS * 2 * C::A_BYTES;
          const uint32_t be_hi = bb, bo_hi = bb + C::BE_BYTES;
          const uint32_t be_lo = bb + C::BE_BYTES + C::BO_BYTES, bo_lo = be_lo + C::BE_BYTES;
#pragma unroll
          for (int ks = 0; ks < CK / 8; ++ks) {
            const uint32_t acc = (c > 0 || ks > 0) ? 1u : 0u;
            const uint32_t o = ks * 256;
            umma_tf32(tmem, umma_sdesc(ae_hi + o, 128, C::SBO), umma_sdesc(be_hi + o, 128, C::SBO), ide, acc);
            if constexpr (PASSES == 3) {
              umma_tf32(tmem, umma_sdesc(ae_hi + o, 128, C::SBO), umma_sdesc(be_lo + o, 128, C::SBO), ide, 1u);
              umma_tf32(tmem, umma_sdesc(ae_lo + o, 128, C::SBO), umma_sdesc(be_hi + o, 128, C::SBO), ide, 1u);
            }
            if (c < C::CO) {
              umma_tf32(tmem + C::NBE, umma_sdesc(ao_hi + o, 128, C::SBO), umma_sdesc(bo_hi + o, 128, C::SBO), ido,
                        acc);
              if constexpr (PASSES == 3) {
                umma_tf32(tmem + C::NBE, umma_sdesc(ao_hi + o, 128, C::SBO), umma_sdesc(bo_lo + o, 128, C::SBO),
                          ido, 1u);
                umma_tf32(tmem + C::NBE, umma_sdesc(ao_lo + o, 128, C::SBO), umma_sdesc(bo_hi + o, 128, C::SBO),
                          ido, 1u);
              }
            }
          }
          umma_commit(&empty[s]);  // the stage is free once these MMAs have read it
        }
        if (*s_abort) break;
        umma_commit(acc_full);
      }
      umma_commit(fin);
      if (!mbar_wait_bounded(fin, 0)) fail();
    }
  } else if (warp < 4) {
    // ---- epilogue: TMEM lane = row = patch ----------------------------------------
    const int m = tid;
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
  (void)N1;
}

}  // namespace tps
