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
// evaluated with the interior of x set to zero, which turns the 49 interior
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
//    one 1D line per thread in registers, applies the centro-symmetric 1D
//    matrices in even/odd folded form (constant-bank operands, about half the
//    multiply-adds), and the last one stores x_I straight to global memory;
//  * a second loader variant (plain coalesced loads) serves vectors whose
//    pitch is not 16-byte aligned (the C-ABI level operations on caller
//    vectors); the compute path is shared.
#pragma once

#include <cuda.h>

#include "ptx.cuh"
#include "smoother.cuh"
#include "tps_common.cuh"

namespace tps {

template <int K, typename T>
struct Sm3 {
  static constexpr int N1 = 2 * K + 1, M = 2 * K - 1;
  static constexpr int A = 16 / static_cast<int>(sizeof(T));  // TMA x-alignment (elements)
  static constexpr int W = ((N1 + A - 1) + A - 1) / A * A;    // staged row width
  static constexpr int XBOX = N1 * N1 * W;
  static constexpr int BBOX = M * M * W;
  static constexpr int ALIGN = 128 / static_cast<int>(sizeof(T));  // TMA destinations: 128 B
  static constexpr int VSZ = M * M * N1;   // zy-contracted [zi][yi][x]
  // the x box region also holds V1/V2 once the z stage is done
  static constexpr int XREG = XBOX > 2 * VSZ ? XBOX : 2 * VSZ;
  static constexpr int BOFF = (XREG + ALIGN - 1) / ALIGN * ALIGN;    // b slab inside a stage
  static constexpr int STAGE = (BOFF + BBOX + ALIGN - 1) / ALIGN * ALIGN;  // per patch
  static constexpr int ZSZ = M * N1 * N1;  // z-contracted  [zi][y][x]
  static constexpr int QSZ = M * M * M;
  static constexpr int RING = N1 * N1 - M * M;  // boundary lines of a z-face
  // patches per batch: enough lines per stage, two CTAs per SM within 227 KB
  static constexpr int PPB = sizeof(T) == 4 ? (K == 1 ? 32 : K == 2 ? 16 : K == 3 ? 8 : K == 4 ? 4 : K <= 6 ? 2 : 1)
                                            : (K == 1 ? 16 : K == 2 ? 8 : K == 3 ? 4 : K == 4 ? 2 : 1);
  static constexpr int NT_RAW = (PPB * M * M + 31) / 32 * 32;
  static constexpr int NT = NT_RAW < 128 ? 128 : NT_RAW;
  // shared memory layout (elements of T): 2 stages | Z1 | Z2 | 1/(lambda sums) ;
  // V1/V2 of a patch live in the x box of its own stage (dead after the z stage),
  // Q1/Q2 alias Z1/Z2
  static_assert(2 * VSZ <= BOFF, "V arrays must fit in the staged x box");
  static constexpr int OFF_Z1 = 2 * PPB * STAGE;
  static constexpr int OFF_Z2 = OFF_Z1 + PPB * ZSZ;
  static constexpr int OFF_RL = OFF_Z2 + PPB * ZSZ;
  static constexpr int ELEMS = (OFF_RL + QSZ + ALIGN - 1) / ALIGN * ALIGN;
  // + two mbarriers and the wait-status flag
  static constexpr size_t BYTES = sizeof(T) * ELEMS + 2 * sizeof(uint64_t) + 16;
};

// out[0..M) = interior rows 1..M of A v for a centro-symmetric (2k+1)^2 patch
// matrix, from the folded input e[j] = v_j + v_{2k-j}, o[j] = v_j - v_{2k-j}
// (j < k), e[k] = v_k.
template <int K, typename T>
__device__ __forceinline__ void fold_rows(const T *fe, const T *fo, const T (&e)[K + 1],
                                          const T (&o)[K > 1 ? K : 1], T (&out)[2 * K - 1])
{
  constexpr int M = 2 * K - 1;
#pragma unroll
  for (int r = 0; r < K - 1; ++r) {
    T se = fe[r * (K + 1) + K] * e[K];
    T so = T(0);
#pragma unroll
    for (int j = 0; j < K; ++j) {
      se += fe[r * (K + 1) + j] * e[j];
      so += fo[r * K + j] * o[j];
    }
    out[r] = se + so;
    out[M - 1 - r] = se - so;
  }
  T sc = fe[(K - 1) * (K + 1) + K] * e[K];
#pragma unroll
  for (int j = 0; j < K; ++j) sc += fe[(K - 1) * (K + 1) + j] * e[j];
  out[K - 1] = sc;
}

template <int K, typename T>
__device__ __forceinline__ void fold_in(const T (&v)[2 * K + 1], T (&e)[K + 1], T (&o)[K > 1 ? K : 1])
{
#pragma unroll
  for (int j = 0; j < K; ++j) {
    e[j] = v[j] + v[2 * K - j];
    o[j] = v[j] - v[2 * K - j];
  }
  e[K] = v[K];
}

struct Sm3Args {
  int nx_c, ny_c, n_patches;  // patch lattice of the colour
  int cx, cy, cz;             // colour parities
  int n_batches;
  int zero_x;                 // x == 0 on entry (first colour of a zero-initialised sweep)
  int64_t sy, sz;             // vector pitches (elements)
};

template <int K, typename T, bool USE_TMA>
__global__ void __launch_bounds__(Sm3<K, T>::NT)
    smoother3d_kernel(const __grid_constant__ CUtensorMap map_x,
                      const __grid_constant__ CUtensorMap map_b, T *__restrict__ x,
                      const T *__restrict__ b, const Sm3Args a, T scale, T fd_scale,
                      int *__restrict__ err)
{
  using S = Sm3<K, T>;
  constexpr int N1 = S::N1, M = S::M, W = S::W, PPB = S::PPB, NT = S::NT, AL = S::A;
  const DegreeTables<K, T> &tb = c_tables<K, T>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T *sm = reinterpret_cast<T *>(smem_raw);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + sizeof(T) * S::ELEMS);
  int &s_ok = *reinterpret_cast<int *>(bars + 2);
  const int tid = threadIdx.x;

  // patch j of the colour -> first DoF coordinates of its box
  auto patch_xyz = [&](int j, int &fx, int &fy, int &fz) {
    const int jx = j % a.nx_c, jy = (j / a.nx_c) % a.ny_c, jz = j / (a.nx_c * a.ny_c);
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
    uint32_t bytes = 0;
    const int np = min(PPB, a.n_patches - bt * PPB);
    bytes = np * sizeof(T) * (S::BBOX + (a.zero_x ? 0 : S::XBOX));
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

    // x offset of each patch's box inside its staged rows
    auto xoff = [&](int lp) -> int {
      if constexpr (!USE_TMA) return 0;
      int fx, fy, fz;
      patch_xyz(bt * PPB + (lp < np ? lp : 0), fx, fy, fz);
      return fx & (AL - 1);
    };

    T *Z1 = sm + S::OFF_Z1, *Z2 = sm + S::OFF_Z2;
    // V1/V2 of patch lp at stage + lp*STAGE (+VSZ): the x box is dead after the z stage
    T *V1 = stage, *V2 = stage + S::VSZ;
    constexpr int VST = S::STAGE;  // V1/V2 patch stride
    T *Q1 = Z1, *Q2 = Z2;  // the fast-diagonalization stages reuse the Z arrays

    if (!a.zero_x) {
      // ---- z: Z1 = M_z x~, Z2 = L_z x~ (x~ = x with zero interior) ----------
      // ring lines (y or x on the box boundary) first, then interior lines
      for (int t = tid; t < PPB * N1 * N1; t += NT) {
        int lp, y, xx;
        const bool ring = t < PPB * S::RING;
        if (ring) {
          lp = t / S::RING;
          const int r = t % S::RING;
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
        } else {
          const int u = t - PPB * S::RING;
          lp = u / (M * M);
          const int r = u % (M * M);
          y = 1 + r / M;
          xx = 1 + r % M;
        }
        const T *src = stage + lp * S::STAGE + y * W + xoff(lp) + xx;
        T *d1 = Z1 + lp * S::ZSZ + y * N1 + xx, *d2 = Z2 + lp * S::ZSZ + y * N1 + xx;
        if (ring) {
          T v[N1], e[K + 1], o[K > 1 ? K : 1], r1[M], r2[M];
#pragma unroll
          for (int z = 0; z < N1; ++z) v[z] = src[z * N1 * W];
          fold_in<K, T>(v, e, o);
          fold_rows<K, T>(tb.pmass_fe, tb.pmass_fo, e, o, r1);
          fold_rows<K, T>(tb.plap_fe, tb.plap_fo, e, o, r2);
#pragma unroll
          for (int i = 0; i < M; ++i) {
            d1[i * N1 * N1] = r1[i];
            d2[i * N1 * N1] = r2[i];
          }
        } else {
          const T v0 = src[0], vn = src[(N1 - 1) * N1 * W];
#pragma unroll
          for (int i = 0; i < M; ++i) {
            d1[i * N1 * N1] = tb.pmass[(i + 1) * N1] * v0 + tb.pmass[(i + 1) * N1 + N1 - 1] * vn;
            d2[i * N1 * N1] = tb.plap[(i + 1) * N1] * v0 + tb.plap[(i + 1) * N1 + N1 - 1] * vn;
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
        T v[N1], e1[K + 1], o1[K > 1 ? K : 1], e2[K + 1], o2[K > 1 ? K : 1];
#pragma unroll
        for (int j = 0; j < N1; ++j) v[j] = s1[j * N1];
        fold_in<K, T>(v, e1, o1);
#pragma unroll
        for (int j = 0; j < N1; ++j) v[j] = s2[j * N1];
        fold_in<K, T>(v, e2, o2);
        T ra[M], rb[M], rc[M];
        fold_rows<K, T>(tb.pmass_fe, tb.pmass_fo, e2, o2, ra);
        fold_rows<K, T>(tb.plap_fe, tb.plap_fo, e1, o1, rb);
        fold_rows<K, T>(tb.pmass_fe, tb.pmass_fo, e1, o1, rc);
        T *d1 = V1 + lp * VST + zi * M * N1 + xx, *d2 = V2 + lp * VST + zi * M * N1 + xx;
#pragma unroll
        for (int i = 0; i < M; ++i) {
          d1[i * N1] = ra[i] + rb[i];
          d2[i * N1] = rc[i];
        }
      }
      __syncthreads();
    }
    // ---- x: r = b - s (M_x V1 + L_x V2), then S^T along x -> Q1 -----------
    for (int t = tid; t < PPB * M * M; t += NT) {
      const int lp = t / (M * M), r = t % (M * M);  // r = zi * M + yi
      T res[M];
      const T *bb = stage + lp * S::STAGE + S::BOFF + r * W + xoff(lp) + 1;
      if (!a.zero_x) {
        const T *s1 = V1 + lp * VST + r * N1, *s2 = V2 + lp * VST + r * N1;
        T v[N1], e1[K + 1], o1[K > 1 ? K : 1], e2[K + 1], o2[K > 1 ? K : 1];
#pragma unroll
        for (int j = 0; j < N1; ++j) v[j] = s1[j];
        fold_in<K, T>(v, e1, o1);
#pragma unroll
        for (int j = 0; j < N1; ++j) v[j] = s2[j];
        fold_in<K, T>(v, e2, o2);
        T ra[M], rb[M];
        fold_rows<K, T>(tb.pmass_fe, tb.pmass_fo, e1, o1, ra);
        fold_rows<K, T>(tb.plap_fe, tb.plap_fo, e2, o2, rb);
#pragma unroll
        for (int i = 0; i < M; ++i) res[i] = bb[i] - scale * (ra[i] + rb[i]);
      } else {
#pragma unroll
        for (int i = 0; i < M; ++i) res[i] = bb[i];
      }
      T q[M];
      apply_evec<K, T, true>(res, q);
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
      apply_evec<K, T, true>(v, q);
      T *d = Q2 + lp * S::QSZ + zi * M * M + qx;
#pragma unroll
      for (int j = 0; j < M; ++j) d[j * M] = q[j];
    }
    __syncthreads();
    // ---- S^T along z, eigenvalue scaling, S along z: Q2 -> Q1 ---------------
    for (int t = tid; t < PPB * M * M; t += NT) {
      const int lp = t / (M * M), r = t % (M * M);
      const int qy = r / M, qx = r % M;
      const T *s = Q2 + lp * S::QSZ + r;
      T v[M], q[M];
#pragma unroll
      for (int j = 0; j < M; ++j) v[j] = s[j * M * M];
      apply_evec<K, T, true>(v, q);
#pragma unroll
      for (int j = 0; j < M; ++j) q[j] *= RL[j * M * M + r];
      apply_evec<K, T, false>(q, v);
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
      apply_evec<K, T, false>(v, q);
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
      apply_evec<K, T, false>(v, q);
      if (lp < np) {
        int fx, fy, fz;
        patch_xyz(bt * PPB + lp, fx, fy, fz);
        T *dst = x + (fx + 1 + xx) + (fy + 1) * a.sy + (fz + 1 + z) * a.sz;
#pragma unroll
        for (int j = 0; j < M; ++j) dst[j * a.sy] = q[j];
      }
    }
    __syncthreads();  // every read of this stage is done before it is refilled
  }
}

}  // namespace tps
