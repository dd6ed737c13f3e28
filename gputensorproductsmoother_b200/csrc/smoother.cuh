// Fused vertex-patch smoother kernel (one launch per colour), sm_100a; used
// for 2D levels (3D levels use smoother3d.cuh).
//
// Reference behaviour: LevelVertexPatch::patch_loop_fused + loop_kernel_fused_cf
// / loop_kernel_fused_l (include/patch_base.template.cuh:379-543,
// include/loop_kernel.cuh:786-884, 962-1060) with LocalSmoother<FUSED_CF/L>
// (include/evaluate_kernel.cuh:1890-1971, 2058-2163): for every patch p of the
// colour,  x_I(p) <- omega * (x_I(p) + A_II^{-1} (b - A_p x)_I).
//
// B200 design:
//  * patches of a colour are enumerated arithmetically (stride-2 lattice of
//    vertices), no first_dof/patch_id index arrays;
//  * each CTA stages the (2k+1)^d boxes of PPB patches in shared memory, the
//    residual is evaluated only on the (2k-1)^d interior rows (7 1D
//    contractions in 3D, interior-row outputs), b is read only on the interior;
//  * all 1D tables are immediate constant-bank operands of fully unrolled FMA
//    chains; each thread owns one 1D line and keeps it in registers
//    (n1 loads feed 2m outputs);
//  * the fast-diagonalization factors are exactly even/odd (host FP64
//    eigensolver), so S^T and S are applied on the folded half-lines:
//    ~half the multiply-adds of a dense m x m contraction;
//  * the result is written straight from the registers of the last
//    contraction (coalesced along x).
#pragma once

#include "tps_common.cuh"

namespace tps {

template <int DIM, int K>
struct SmootherShape {
  static constexpr int N1 = Dims<K>::N1, M = Dims<K>::M;
  static constexpr int BOX = DIM == 3 ? N1 * N1 * N1 : N1 * N1;
  static constexpr int INT = DIM == 3 ? M * M * M : M * M;
  static constexpr int TSZ = DIM == 3 ? N1 * N1 * M : N1 * M;  // x-contracted
  static constexpr int USZ = DIM == 3 ? N1 * M * M : 0;        // xy-contracted
  static constexpr int PER_PATCH = BOX + INT + 2 * TSZ + 2 * USZ;
  static constexpr int LINES = DIM == 3 ? N1 * N1 : N1;
  // patches per CTA and threads per CTA (tuned for the 148-SM B200)
  static constexpr int PPB = DIM == 3 ? (K == 1 ? 16 : K == 2 ? 5 : K == 3 ? 3 : K == 4 ? 2 : 1)
                                      : (K <= 2 ? 16 : K <= 4 ? 8 : 4);
  static constexpr int NT = DIM == 3 ? (K <= 5 ? 128 : K == 6 ? 192 : 256) : 128;
};

// Apply the fast-diagonalization factor S (eigenvectors as columns) or S^T
// to a line of M values held in registers.  The host orders the modes so that
// columns 0..C (C = k-1, the centre index) are the reflection-even
// eigenvectors and columns C+1..M-1 the odd ones; both products are then
// evaluated on folded half-lines with compile-time parity:
//   S^T: out[q] = sum_j S[j][q] (in_j +/- in_{M-1-j})   (half the MACs)
//   S  : out[i], out[M-1-i] = (even part) +/- (odd part)
template <int K, typename T, bool TRANSPOSE>
__device__ __forceinline__ void apply_evec(const T (&in)[Dims<K>::M], T (&out)[Dims<K>::M])
{
  constexpr int M = Dims<K>::M, C = K - 1;
  const DegreeTables<K, T> &tb = c_tables<K, T>;
  if constexpr (TRANSPOSE) {
    T e[C + 1], o[C > 0 ? C : 1];
#pragma unroll
    for (int j = 0; j < C; ++j) {
      e[j] = in[j] + in[M - 1 - j];
      o[j] = in[j] - in[M - 1 - j];
    }
    e[C] = in[C];
#pragma unroll
    for (int q = 0; q <= C; ++q) {
      T s = tb.evec[C * M + q] * e[C];
#pragma unroll
      for (int j = 0; j < C; ++j) s += tb.evec[j * M + q] * e[j];
      out[q] = s;
    }
#pragma unroll
    for (int q = C + 1; q < M; ++q) {
      T s = T(0);
#pragma unroll
      for (int j = 0; j < C; ++j) s += tb.evec[j * M + q] * o[j];
      out[q] = s;
    }
  } else {
#pragma unroll
    for (int i = 0; i < C; ++i) {
      T se = T(0), so = T(0);
#pragma unroll
      for (int q = 0; q <= C; ++q) se += tb.evec[i * M + q] * in[q];
#pragma unroll
      for (int q = C + 1; q < M; ++q) so += tb.evec[i * M + q] * in[q];
      out[i] = se + so;
      out[M - 1 - i] = se - so;
    }
    T sc = T(0);
#pragma unroll
    for (int q = 0; q <= C; ++q) sc += tb.evec[C * M + q] * in[q];
    out[C] = sc;
  }
}

template <int DIM, int K, typename T>
__global__ void __launch_bounds__(SmootherShape<DIM, K>::NT)
    smoother_colour_kernel(T *__restrict__ x, const T *__restrict__ b, int64_t sy, int64_t sz,
                           int nx_c, int ny_c, int n_patches_c, int cx, int cy, int cz, T scale,
                           T inv_scale, T omega)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  using S = SmootherShape<DIM, K>;
  constexpr int N1 = S::N1, M = S::M, PPB = S::PPB, NT = S::NT;
  const DegreeTables<K, T> &tb = c_tables<K, T>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T *smem = reinterpret_cast<T *>(smem_raw);

  const int p0 = blockIdx.x * PPB;

  // first DoF of local patch lp (include/patch_base.template.cuh:1371-1397)
  auto first_dof = [&](int lp, bool &valid) -> int64_t {
    const int j = p0 + lp;
    valid = j < n_patches_c;
    const int jj = valid ? j : 0;
    const int jx = jj % nx_c;
    const int jy = DIM == 3 ? (jj / nx_c) % ny_c : jj / nx_c;
    const int jz = DIM == 3 ? jj / (nx_c * ny_c) : 0;
    const int px = cx + 2 * jx, py = cy + 2 * jy, pz = DIM == 3 ? cz + 2 * jz : 0;
    return static_cast<int64_t>(px) * K + static_cast<int64_t>(py) * K * sy +
           static_cast<int64_t>(pz) * K * sz;
  };

  T *Xs = smem;                          // PPB * BOX
  T *Bs = Xs + PPB * S::BOX;             // PPB * INT
  T *T1 = Bs + PPB * S::INT;             // PPB * TSZ
  T *T2 = T1 + PPB * S::TSZ;             // PPB * TSZ
  T *U1 = T2 + PPB * S::TSZ;             // PPB * USZ (3D)
  T *U2 = U1 + PPB * S::USZ;             // PPB * USZ (3D)

  // ---- stage 0: gather boxes of x and interiors of b --------------------
  for (int e = threadIdx.x; e < PPB * S::BOX; e += NT) {
    const int lp = e / S::BOX, l = e % S::BOX;
    bool valid;
    const int64_t f = first_dof(lp, valid);
    const int lx = l % N1, ly = (l / N1) % N1, lz = DIM == 3 ? l / (N1 * N1) : 0;
    Xs[e] = valid ? x[f + lx + ly * sy + lz * sz] : T(0);
  }
  for (int e = threadIdx.x; e < PPB * S::INT; e += NT) {
    const int lp = e / S::INT, l = e % S::INT;
    bool valid;
    const int64_t f = first_dof(lp, valid);
    const int lx = l % M + 1, ly = (l / M) % M + 1, lz = DIM == 3 ? l / (M * M) + 1 : 0;
    Bs[e] = valid ? __ldg(&b[f + lx + ly * sy + lz * sz]) : T(0);
  }
  __syncthreads();

  // ---- stage 1: contract x with M and L on interior rows ----------------
  for (int t = threadIdx.x; t < PPB * S::LINES; t += NT) {
    const int lp = t / S::LINES, line = t % S::LINES;
    const T *src = Xs + lp * S::BOX + line * N1;
    T v[N1];
#pragma unroll
    for (int j = 0; j < N1; ++j) v[j] = src[j];
    T *d1 = T1 + lp * S::TSZ + line * M, *d2 = T2 + lp * S::TSZ + line * M;
#pragma unroll
    for (int i = 0; i < M; ++i) {
      T a = T(0), c = T(0);
#pragma unroll
      for (int j = 0; j < N1; ++j) {
        a += tb.pmass[(i + 1) * N1 + j] * v[j];
        c += tb.plap[(i + 1) * N1 + j] * v[j];
      }
      d1[i] = a;
      d2[i] = c;
    }
  }
  __syncthreads();

  T *R = T1;  // interior residual (T1 is dead after the y stage)
  if constexpr (DIM == 3) {
    // ---- stage 2: contract y: U1 = M_y T1, U2 = L_y T1 + M_y T2 ----------
    for (int t = threadIdx.x; t < PPB * N1 * M; t += NT) {
      const int lp = t / (N1 * M), r = t % (N1 * M);
      const int z = r / M, xx = r % M;
      const T *s1 = T1 + lp * S::TSZ + z * N1 * M + xx;
      const T *s2 = T2 + lp * S::TSZ + z * N1 * M + xx;
      T a[N1], c[N1];
#pragma unroll
      for (int j = 0; j < N1; ++j) {
        a[j] = s1[j * M];
        c[j] = s2[j * M];
      }
      T *d1 = U1 + lp * S::USZ + z * M * M + xx, *d2 = U2 + lp * S::USZ + z * M * M + xx;
#pragma unroll
      for (int i = 0; i < M; ++i) {
        T u1 = T(0), u2 = T(0);
#pragma unroll
        for (int j = 0; j < N1; ++j) {
          u1 += tb.pmass[(i + 1) * N1 + j] * a[j];
          u2 += tb.plap[(i + 1) * N1 + j] * a[j] + tb.pmass[(i + 1) * N1 + j] * c[j];
        }
        d1[i * M] = u1;
        d2[i * M] = u2;
      }
    }
    __syncthreads();
    // ---- stage 3: contract z and form r = b - s (L_z U1 + M_z U2) --------
    for (int t = threadIdx.x; t < PPB * M * M; t += NT) {
      const int lp = t / (M * M), yx = t % (M * M);
      const T *s1 = U1 + lp * S::USZ + yx, *s2 = U2 + lp * S::USZ + yx;
      T a[N1], c[N1];
#pragma unroll
      for (int j = 0; j < N1; ++j) {
        a[j] = s1[j * M * M];
        c[j] = s2[j * M * M];
      }
      const T *bb = Bs + lp * S::INT + yx;
      T *rr = R + lp * S::TSZ + yx;
#pragma unroll
      for (int i = 0; i < M; ++i) {
        T acc = T(0);
#pragma unroll
        for (int j = 0; j < N1; ++j)
          acc += tb.plap[(i + 1) * N1 + j] * a[j] + tb.pmass[(i + 1) * N1 + j] * c[j];
        rr[i * M * M] = bb[i * M * M] - scale * acc;
      }
    }
    __syncthreads();
  } else {
    // ---- 2D stage 2: contract y and form r = b - s (L_y T1 + M_y T2) ------
    for (int t = threadIdx.x; t < PPB * M; t += NT) {
      const int lp = t / M, xx = t % M;
      const T *s1 = T1 + lp * S::TSZ + xx, *s2 = T2 + lp * S::TSZ + xx;
      T a[N1], c[N1];
#pragma unroll
      for (int j = 0; j < N1; ++j) {
        a[j] = s1[j * M];
        c[j] = s2[j * M];
      }
      T res[M];
      const T *bb = Bs + lp * S::INT + xx;
#pragma unroll
      for (int i = 0; i < M; ++i) {
        T acc = T(0);
#pragma unroll
        for (int j = 0; j < N1; ++j)
          acc += tb.plap[(i + 1) * N1 + j] * a[j] + tb.pmass[(i + 1) * N1 + j] * c[j];
        res[i] = bb[i * M] - scale * acc;
      }
      // each thread reads and writes only its own column xx of T1/R
#pragma unroll
      for (int i = 0; i < M; ++i) R[lp * S::TSZ + i * M + xx] = res[i];
    }
    __syncthreads();
  }

  // ---- fast diagonalization on the interior --------------------------------
  // ping-pong between R (in T1) and Q (in T2)
  T *Q = T2;
  constexpr int LINES_I = DIM == 3 ? M * M : M;  // lines per direction
  // S^T along x: R -> Q
  for (int t = threadIdx.x; t < PPB * LINES_I; t += NT) {
    const int lp = t / LINES_I, line = t % LINES_I;
    T in[M], out[M];
    const T *s = R + lp * S::TSZ + line * M;
#pragma unroll
    for (int j = 0; j < M; ++j) in[j] = s[j];
    apply_evec<K, T, true>(in, out);
    T *d = Q + lp * S::TSZ + line * M;
#pragma unroll
    for (int j = 0; j < M; ++j) d[j] = out[j];
  }
  __syncthreads();
  // S^T along y: Q -> R   (3D: lines indexed by (z, x); 2D: by x)
  for (int t = threadIdx.x; t < PPB * LINES_I; t += NT) {
    const int lp = t / LINES_I, line = t % LINES_I;
    const int z = DIM == 3 ? line / M : 0, xx = line % M;
    const int base = z * M * M + xx;
    T in[M], out[M];
    const T *s = Q + lp * S::TSZ + base;
#pragma unroll
    for (int j = 0; j < M; ++j) in[j] = s[j * M];
    apply_evec<K, T, true>(in, out);
    T *d = R + lp * S::TSZ + base;
    if constexpr (DIM == 2) {
      // divide by lambda_x + lambda_y, scaled back to physical cells
#pragma unroll
      for (int j = 0; j < M; ++j) d[j * M] = out[j] * inv_scale / (tb.eval[xx] + tb.eval[j]);
    } else {
#pragma unroll
      for (int j = 0; j < M; ++j) d[j * M] = out[j];
    }
  }
  __syncthreads();
  if constexpr (DIM == 3) {
    // S^T along z with the eigenvalue division: R -> Q
    for (int t = threadIdx.x; t < PPB * M * M; t += NT) {
      const int lp = t / (M * M), yx = t % (M * M);
      const int yy = yx / M, xx = yx % M;
      T in[M], out[M];
      const T *s = R + lp * S::TSZ + yx;
#pragma unroll
      for (int j = 0; j < M; ++j) in[j] = s[j * M * M];
      apply_evec<K, T, true>(in, out);
      T *d = Q + lp * S::TSZ + yx;
      const T lxy = tb.eval[xx] + tb.eval[yy];
#pragma unroll
      for (int j = 0; j < M; ++j) d[j * M * M] = out[j] * inv_scale / (lxy + tb.eval[j]);
    }
    __syncthreads();
  }
  T *V = DIM == 3 ? Q : R;  // divided coefficients
  T *W = DIM == 3 ? R : Q;
  // S along x: V -> W
  for (int t = threadIdx.x; t < PPB * LINES_I; t += NT) {
    const int lp = t / LINES_I, line = t % LINES_I;
    T in[M], out[M];
    const T *s = V + lp * S::TSZ + line * M;
#pragma unroll
    for (int j = 0; j < M; ++j) in[j] = s[j];
    apply_evec<K, T, false>(in, out);
    T *d = W + lp * S::TSZ + line * M;
#pragma unroll
    for (int j = 0; j < M; ++j) d[j] = out[j];
  }
  __syncthreads();
  if constexpr (DIM == 3) {
    // S along y: W -> V
    for (int t = threadIdx.x; t < PPB * M * M; t += NT) {
      const int lp = t / (M * M), r = t % (M * M);
      const int z = r / M, xx = r % M;
      const int base = z * M * M + xx;
      T in[M], out[M];
      const T *s = W + lp * S::TSZ + base;
#pragma unroll
      for (int j = 0; j < M; ++j) in[j] = s[j * M];
      apply_evec<K, T, false>(in, out);
      T *d = V + lp * S::TSZ + base;
#pragma unroll
      for (int j = 0; j < M; ++j) d[j * M] = out[j];
    }
    __syncthreads();
    // S along z and write x_I = omega (x_I + delta)
    for (int t = threadIdx.x; t < PPB * M * M; t += NT) {
      const int lp = t / (M * M), yx = t % (M * M);
      bool valid;
      const int64_t f = first_dof(lp, valid);
      T in[M], out[M];
      const T *s = V + lp * S::TSZ + yx;
#pragma unroll
      for (int j = 0; j < M; ++j) in[j] = s[j * M * M];
      apply_evec<K, T, false>(in, out);
      if (valid) {
        const int yy = yx / M, xx = yx % M;
        const T *xb = Xs + lp * S::BOX + (yy + 1) * N1 + xx + 1;
        T *xg = x + f + (xx + 1) + (yy + 1) * sy;
#pragma unroll
        for (int j = 0; j < M; ++j) xg[(j + 1) * sz] = omega * (xb[(j + 1) * N1 * N1] + out[j]);
      }
    }
  } else {
    // 2D: S along y and write
    for (int t = threadIdx.x; t < PPB * M; t += NT) {
      const int lp = t / M, xx = t % M;
      bool valid;
      const int64_t f = first_dof(lp, valid);
      T in[M], out[M];
      const T *s = W + lp * S::TSZ + xx;
#pragma unroll
      for (int j = 0; j < M; ++j) in[j] = s[j * M];
      apply_evec<K, T, false>(in, out);
      if (valid) {
        const T *xb = Xs + lp * S::BOX + N1 + xx + 1;
        T *xg = x + f + (xx + 1);
#pragma unroll
        for (int j = 0; j < M; ++j) xg[(j + 1) * sy] = omega * (xb[j * N1] + out[j]);
      }
    }
  }
}

}  // namespace tps
