// 3D matrix-free Laplace operator, z-marching form with two output columns
// per thread (sm_100a).
//
// Reference behaviour: LaplaceOperator::vmult (include/laplace_operator.cuh:86-101)
// and the residual b - A x of the V-cycle.  Algebra as in laplace.cuh: on the
// uniform tensor mesh A = s (L_z M_y M_x + M_z L_y M_x + M_z M_y L_x) with the
// banded global 1D mass and stiffness matrices, applied as two x products,
// three y products and two z products (~42 multiply-adds per DoF).
//
// Layout for few instructions per DoF (the operator is bound by instruction
// issue, not by its 2 x 8 bytes of HBM traffic per DoF):
// * a CTA owns TX x TY cells in x, y and marches through a range of cell
//   layers in z; the input planes of a layer (its tile plus a one-cell xy
//   halo) are copied global -> shared by cp.async with zero fill outside the
//   mesh -- no register staging -- and the next layer's copy runs while the
//   current layer is contracted in y and z;
// * x stage: one thread per (plane, row, cell) reads the 2k+1 inputs of a
//   cell segment with 16-byte shared loads and writes the k outputs of M_x
//   and L_x;
// * y and z stages: one thread per pair of adjacent x columns, so every
//   shared access moves two values and every coefficient serves both columns
//   (one packed fma.rn.f32x2 per coefficient in FP32);
// * z stage: the (k+1) x (k+1) cell matrices act on the k+1 xy-contracted
//   planes of a cell layer: the k new ones in shared slots, the vertex plane
//   shared with the previous layer in the owning thread's registers; the
//   output plane shared with the next layer is carried in registers too.  A
//   CTA starts one layer early to form both carries.
// * every thread's task offsets are fixed for the whole march (the stages'
//   task counts are multiples of, or at most, the thread count).
// Row pitches and slot strides are padded so that the shared accesses of
// all three stages are (nearly) free of bank conflicts (wavefront model of the
// thread mappings below).  Three barriers per cell layer.  Deterministic: no
// atomics, every output written once by one thread.
#pragma once

#include "laplace.cuh"
#include "ptx.cuh"
#include "tps_common.cuh"

namespace tps {

// padded pitches {staged row, x-contracted row, extra elements per plane slot}
// per degree, FP64 and FP32 (chosen with a shared-memory wavefront model of
// the three stages' accesses)
constexpr int kMarchPitch64[8][3] = {{0, 0, 0},   {18, 16, 0}, {20, 16, 0}, {20, 20, 12},
                                     {22, 18, 0}, {18, 10, 6}, {20, 20, 12}, {22, 26, 10}};
constexpr int kMarchPitch32[8][3] = {{0, 0, 0},    {18, 16, 0}, {24, 16, 16}, {20, 28, 28},
                                     {24, 16, 16}, {18, 10, 6}, {20, 20, 28}, {22, 14, 10}};

constexpr int march_align4(int x) { return (x + 3) / 4 * 4; }

template <int K, typename T>
struct OpMarch {
  static constexpr int TX = K == 1 ? 16 : K == 2 ? 8 : K <= 4 ? 4 : 2, TY = TX;  // cells per CTA in x, y
  static constexpr int OX = TX * K, OY = TY * K, HX = OX / 2;  // output tile; column pairs per row
  static constexpr int WX = (TX + 1) * K + 1, WY = (TY + 1) * K + 1;  // staged plane (tile + halo)
  static constexpr int VMAX = 16 / int(sizeof(T));
  static constexpr int VX = K % VMAX == 0 ? VMAX : K % 2 == 0 ? 2 : 1;  // x-stage vector width
  static constexpr const int *PITCH = sizeof(T) == 8 ? kMarchPitch64[K] : kMarchPitch32[K];
  static constexpr int BW = PITCH[0], XP = PITCH[1];
  static constexpr int PL = WY * BW;                  // one staged plane
  static constexpr int XS = WY * XP;                  // one x-contracted plane (per product)
  static constexpr int TS = OY * OX + PITCH[2];       // one plane slot (per product)
  static constexpr int NXT = K * WY * TX;             // x-stage tasks per layer
  static constexpr int NYT = K * HX * TY;             // y-stage tasks per layer
  static constexpr int NZT = OY * HX;                 // z-stage column pairs
  static constexpr int NT = ((NYT > NZT ? NYT : NZT) + 31) / 32 * 32;
  static constexpr int EPT = (WY * WX + NT - 1) / NT;  // staged entries per thread and plane
  static constexpr int CZ = 16;                        // cell layers per CTA (the default's most)
  // shared memory (elements): IN[K][PL] | X1[K][XS] | X2[K][XS] | T1[K][TS] | T2[K][TS]
  static constexpr int OFF_X1 = march_align4(K * PL);
  static constexpr int OFF_X2 = march_align4(OFF_X1 + K * XS);
  static constexpr int OFF_T1 = march_align4(OFF_X2 + K * XS);
  static constexpr int OFF_T2 = march_align4(OFF_T1 + K * TS);
  static constexpr int ELEMS = OFF_T2 + K * TS;
  static_assert(BW >= WX && BW % VX == 0 && XP >= OX && XP % 2 == 0 && XP % VX == 0, "pitches");
  static_assert(OX % 2 == 0 && TS % 2 == 0, "column pairs");
};

// CTAs per SM the registers must allow (no spills at these caps; the FP64
// residual holds b of the layer's outputs as well and needs 168 registers at
// degree 4; the fused dot fits 128, with 125: measured, 3D Q4 64^3 mixed
// solve 12.54 -> 12.41 ms with 4 instead of 3 CTAs for it)
template <int K, typename T, OpMode MODE, bool DOT>
constexpr int march_minb()
{
  if constexpr (sizeof(T) == 8) return K <= 3 ? 4 : K == 4 ? (MODE == OpMode::Vmult ? 4 : 3) : 2;
  return K <= 6 ? 4 : 3;
}

template <int K, typename T>
inline int opmarch_layers(int n, int want)
{
  using S = OpMarch<K, T>;
  const int xy = ((n + S::TX - 1) / S::TX) * ((n + S::TY - 1) / S::TY);
  for (int cz = S::CZ; cz > 1; cz /= 2)
    if (xy * ((n + cz - 1) / cz) >= want) return cz;
  return 1;
}

// N consecutive values from 16-byte (VX * sizeof(T)) aligned shared memory
template <int N, int VX, typename T>
__device__ __forceinline__ void march_load_row(const T *p, T (&v)[N])
{
  constexpr int NC = N / VX;
#pragma unroll
  for (int i = 0; i < NC; ++i) {
    if constexpr (VX == 4 && sizeof(T) == 4) {
      const float4 q = *reinterpret_cast<const float4 *>(p + 4 * i);
      v[4 * i] = q.x;
      v[4 * i + 1] = q.y;
      v[4 * i + 2] = q.z;
      v[4 * i + 3] = q.w;
    } else if constexpr (VX == 2) {
      const typename Pair<T>::type q = *reinterpret_cast<const typename Pair<T>::type *>(p + 2 * i);
      v[2 * i] = q.x;
      v[2 * i + 1] = q.y;
    } else {
      v[i] = p[i];
    }
  }
#pragma unroll
  for (int i = NC * VX; i < N; ++i) v[i] = p[i];
}

template <int N, int VX, typename T>
__device__ __forceinline__ void march_store_row(T *p, const T (&v)[N])
{
  static_assert(N % VX == 0, "vector store");
#pragma unroll
  for (int i = 0; i < N / VX; ++i) {
    if constexpr (VX == 4 && sizeof(T) == 4) {
      *reinterpret_cast<float4 *>(p + 4 * i) = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
    } else if constexpr (VX == 2) {
      *reinterpret_cast<typename Pair<T>::type *>(p + 2 * i) = Pair<T>::make(v[2 * i], v[2 * i + 1]);
    } else {
      p[i] = v[i];
    }
  }
}

// entry i of the cell mass (MAT 0) or stiffness (MAT 1) matrix, read from
// the constant bank at an offset fixed at compile time
template <int K, typename T, int MAT>
__device__ __forceinline__ T march_coef(int i)
{
  return MAT == 0 ? c_tables<K, T>.cmass[i] : c_tables<K, T>.clap[i];
}

// k outputs of one cell segment of a global 1D banded product (band_apply of
// laplace.cuh): v[0..2k] = nodes (c-1)k .. (c+1)k
template <int K, typename T, int MAT>
__device__ __forceinline__ void march_band(const T (&v)[2 * K + 1], T (&out)[K])
{
#pragma unroll
  for (int a = 0; a < K; ++a) {
    T s = march_coef<K, T, MAT>(a * (K + 1)) * v[K];
#pragma unroll
    for (int b = 1; b <= K; ++b) s = fmadd(march_coef<K, T, MAT>(a * (K + 1) + b), v[K + b], s);
    if (a == 0) {
#pragma unroll
      for (int b = 0; b <= K; ++b) s = fmadd(march_coef<K, T, MAT>(K * (K + 1) + b), v[b], s);
    }
    out[a] = s;
  }
}

// the same for a pair of columns
template <int K, typename T, int MAT>
__device__ __forceinline__ void march_band2(const typename Pair<T>::type (&v)[2 * K + 1],
                                            typename Pair<T>::type (&out)[K])
{
  using P = Pair<T>;
#pragma unroll
  for (int a = 0; a < K; ++a) {
    T m = march_coef<K, T, MAT>(a * (K + 1));
    typename P::type s = P::fma(P::make(m, m), v[K], P::make(T(0), T(0)));
#pragma unroll
    for (int b = 1; b <= K; ++b) {
      m = march_coef<K, T, MAT>(a * (K + 1) + b);
      s = P::fma(P::make(m, m), v[K + b], s);
    }
    if (a == 0) {
#pragma unroll
      for (int b = 0; b <= K; ++b) {
        m = march_coef<K, T, MAT>(K * (K + 1) + b);
        s = P::fma(P::make(m, m), v[b], s);
      }
    }
    out[a] = s;
  }
}

// x stage over planes 0..NPL-1 of IN: X1 = M_x u, X2 = L_x u (tile columns
// only).  Task t = (row r = plane * WY + y, cell c), t = r * TX + c; NT is a
// multiple of TX, so a thread keeps its cell and advances NT / TX rows per round.
template <int K, typename T, int NPL>
__device__ __forceinline__ void march_stage_x(const T *IN, T *X1, T *X2)
{
  using S = OpMarch<K, T>;
  static_assert(S::NT % S::TX == 0, "x-stage rounds");
  constexpr int ROWS = NPL * S::WY, STEP = S::NT / S::TX, ROUNDS = (ROWS + STEP - 1) / STEP;
  const int c = threadIdx.x % S::TX, r0 = threadIdx.x / S::TX;
  const T *in = IN + r0 * S::BW + c * K;
  T *x1 = X1 + r0 * S::XP + c * K, *x2 = X2 + r0 * S::XP + c * K;
#pragma unroll 1
  for (int i = 0; i < ROUNDS; ++i) {
    if (ROWS % STEP != 0 && i == ROUNDS - 1 && r0 + i * STEP >= ROWS) break;
    T v[2 * K + 1], o1[K], o2[K];
    march_load_row<2 * K + 1, S::VX>(in + i * STEP * S::BW, v);
    march_band<K, T, 0>(v, o1);
    march_band<K, T, 1>(v, o2);
    march_store_row<K, S::VX>(x1 + i * STEP * S::XP, o1);
    march_store_row<K, S::VX>(x2 + i * STEP * S::XP, o2);
  }
}

// y stage of one (column pair, plane, cell row) task: T1 = M_y X1,
// T2 = L_y X1 + M_y X2 for the k rows of the cell row; x and t are the task's
// offsets into X1/X2 and T1/T2
template <int K, typename T>
__device__ __forceinline__ void march_y_task(const T *X1, const T *X2, T *T1, T *T2, int x, int t)
{
  using S = OpMarch<K, T>;
  using V2 = typename Pair<T>::type;
  V2 v[2 * K + 1], o1[K], o2[K];
#pragma unroll
  for (int j = 0; j <= 2 * K; ++j) v[j] = *reinterpret_cast<const V2 *>(X1 + x + j * S::XP);
  march_band2<K, T, 0>(v, o1);
  march_band2<K, T, 1>(v, o2);
#pragma unroll
  for (int a = 0; a < K; ++a) *reinterpret_cast<V2 *>(T1 + t + a * S::OX) = o1[a];
#pragma unroll
  for (int j = 0; j <= 2 * K; ++j) v[j] = *reinterpret_cast<const V2 *>(X2 + x + j * S::XP);
  march_band2<K, T, 0>(v, o1);
#pragma unroll
  for (int a = 0; a < K; ++a) {
    V2 w = o2[a];
    w.x += o1[a].x;
    w.y += o1[a].y;
    *reinterpret_cast<V2 *>(T2 + t + a * S::OX) = w;
  }
}

// DOT (Vmult only): every CTA also forms the sum of src * dst over the
// outputs it writes and stores it to dotp[CTA index]: the p.q of a CG step
// without a second pass over both vectors (fixed summation order)
template <int K, typename T, OpMode MODE, bool DOT>
__global__ void __launch_bounds__(OpMarch<K, T>::NT, march_minb<K, T, MODE, DOT>())
    laplace3d_march_kernel(T *__restrict__ dst, const T *__restrict__ src, const T *__restrict__ rhs, int N1g,
                           int n_cells, int64_t sy, int64_t sz, T scale, int cz, double *__restrict__ dotp)
{
  static_assert(!DOT || MODE == OpMode::Vmult, "the fused dot belongs to q = A p");
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  using S = OpMarch<K, T>;
  using P = Pair<T>;
  using V2 = typename P::type;
  constexpr int NT = S::NT, EPT = S::EPT, WX = S::WX, PL = S::PL, HX = S::HX;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T *sm = reinterpret_cast<T *>(smem_raw);
  T *IN = sm, *X1 = sm + S::OFF_X1, *X2 = sm + S::OFF_X2, *T1 = sm + S::OFF_T1, *T2 = sm + S::OFF_T2;
  const int tid = threadIdx.x;
  const int cx0 = blockIdx.x * S::TX, cy0 = blockIdx.y * S::TY;
  const int gx0 = (cx0 - 1) * K, gy0 = (cy0 - 1) * K;  // staged plane origin
  const int cz_begin = blockIdx.z * cz;
  const int cz_end = min(cz_begin + cz, n_cells);
  const int c_first = cz_begin > 0 ? cz_begin - 1 : 0;  // leading layer: carry only

  // this thread's staged entries (the same xy positions in every plane)
  // (global source, shared destination, source bytes: sizeof(T), or 0 for
  // the zero fill outside the mesh); entries past the plane have no copy
  const T *gsrc[EPT];
  uint32_t sdst[EPT], sbytes[EPT];
  const uint32_t in_s = smem_u32(IN);
#pragma unroll
  for (int j = 0; j < EPT; ++j) {
    const int l = tid + j * NT, lx = l % WX, ly = l / WX;
    const int gx = gx0 + lx, gy = gy0 + ly;
    const bool ok = l < S::WY * WX && gx >= 0 && gx < N1g && gy >= 0 && gy < N1g;
    gsrc[j] = src + (ok ? gx + gy * sy : 0);
    sdst[j] = in_s + uint32_t(sizeof(T)) * uint32_t(l < S::WY * WX ? ly * S::BW + lx : 0);
    sbytes[j] = ok ? uint32_t(sizeof(T)) : 0u;
  }
  constexpr bool kFull = EPT * NT <= S::WY * WX;  // every thread's every entry lies in the plane
  const int jlast = (S::WY * WX - 1 - tid) / NT;    // this thread's last entry in the plane
  // copy planes z0 .. z0+np-1 of the staged tile into IN[0..np-1]
  auto issue = [&](int z0, int np) {
    for (int p = 0; p < np; ++p) {
      const int gz = z0 + p;
      const bool zok = gz >= 0 && gz < N1g;
      const int64_t zo = zok ? gz * sz : 0;
      const uint32_t po = uint32_t(p * PL * sizeof(T));
#pragma unroll
      for (int j = 0; j < EPT; ++j)
        if (kFull || j <= jlast) cp_async_zfill_s<sizeof(T)>(sdst[j] + po, gsrc[j] + zo, zok ? sbytes[j] : 0u);
    }
    cp_async_commit();
  };

  // y-stage task of this thread: t = (cell row cy, plane p, column pair xo2),
  // plane cK+1+p goes to slot p
  const bool ytask = tid < S::NYT;
  const int yx2 = tid % HX, yp = (tid / HX) % K, ycy = tid / (HX * K);
  const int yx = yp * S::XS + ycy * K * S::XP + 2 * yx2, yt = yp * S::TS + ycy * K * S::OX + 2 * yx2;
  // z-stage column pair of this thread
  const bool owner = tid < S::NZT;
  const int xo2 = tid % HX, ty = tid / HX;
  const int zt = ty * S::OX + 2 * xo2;
  const int gx = cx0 * K + 2 * xo2, gy = cy0 * K + ty;
  const bool row_in = owner && gy > 0 && gy < N1g - 1;
  const bool in0 = row_in && gx > 0 && gx < N1g - 1, in1 = row_in && gx + 1 > 0 && gx + 1 < N1g - 1;
  const int64_t gxy = int64_t(gx) + int64_t(gy) * sy;

  // prime: plane c_first*K, xy-contracted into slot 0, kept in registers
  issue(c_first * K, 1);
  cp_async_wait_all();
  __syncthreads();
  march_stage_x<K, T, 1>(IN, X1, X2);
  __syncthreads();
  issue(c_first * K + 1, K);  // the first layer's planes
  if (tid < HX * S::TY) {
    const int x2 = tid % HX, cy = tid / HX;
    march_y_task<K, T>(X1, X2, T1, T2, cy * K * S::XP + 2 * x2, cy * K * S::OX + 2 * x2);
  }
  __syncthreads();
  V2 c1 = P::make(T(0), T(0)), c2 = c1;  // T1, T2 of plane cK at this thread's columns
  if (owner) {
    c1 = *reinterpret_cast<const V2 *>(T1 + zt);
    c2 = *reinterpret_cast<const V2 *>(T2 + zt);
  }

  V2 carry = P::make(T(0), T(0));
  double dsum = 0.0;  // DOT: this thread's src * dst
  for (int c = c_first; c < cz_end; ++c) {
    cp_async_wait_all();
    __syncthreads();  // IN holds planes cK+1..cK+K; X and the slots are free
    march_stage_x<K, T, K>(IN, X1, X2);
    __syncthreads();  // X ready, IN free
    if (c + 1 < cz_end) issue((c + 1) * K + 1, K);  // next layer, overlapped with y and z
    if (ytask) march_y_task<K, T>(X1, X2, T1, T2, yx, yt);
    __syncthreads();  // slots 0..K-1 hold planes cK+1 .. (c+1)K
    const bool store = c >= cz_begin && row_in;
    if (owner) {
      V2 rv[K];  // residual: b at this layer's outputs (DOT: src), loaded before the contraction
      if constexpr (MODE == OpMode::Residual || DOT) {
        const T *vin = DOT ? src : rhs;
#pragma unroll
        for (int a = 0; a < K; ++a) {
          const int gz = c * K + a;
          const bool zin = store && gz > 0 && gz < N1g - 1;
          const T *rp = vin + gxy + int64_t(gz) * sz;
          rv[a].x = zin && in0 ? rp[0] : T(0);
          rv[a].y = zin && in1 ? rp[1] : T(0);
        }
      }
      V2 u1[K + 1], u2[K + 1];
      u1[0] = c1;
      u2[0] = c2;
#pragma unroll
      for (int b = 1; b <= K; ++b) {
        u1[b] = *reinterpret_cast<const V2 *>(T1 + (b - 1) * S::TS + zt);
        u2[b] = *reinterpret_cast<const V2 *>(T2 + (b - 1) * S::TS + zt);
      }
      c1 = u1[K];
      c2 = u2[K];
      // output a of the layer = row a of the cell matrices on the k+1 planes;
      // row 0 adds the previous layer's row k (the shared vertex plane), and
      // row k is carried to the next layer
#pragma unroll
      for (int a = 0; a <= K; ++a) {
        V2 acc = P::make(T(0), T(0));
#pragma unroll
        for (int b = 0; b <= K; ++b) {
          const T l = march_coef<K, T, 1>(a * (K + 1) + b), m = march_coef<K, T, 0>(a * (K + 1) + b);
          acc = P::fma(P::make(l, l), u1[b], acc);
          acc = P::fma(P::make(m, m), u2[b], acc);
        }
        if (a == K) {
          carry = acc;
          break;
        }
        if (a == 0) {
          acc.x += carry.x;
          acc.y += carry.y;
        }
        const int gz = c * K + a;
        if (!store || gz < 1 || gz > N1g - 2) continue;
        T *dp = dst + gxy + int64_t(gz) * sz;
        if constexpr (MODE == OpMode::Vmult) {
          const T q0 = scale * acc.x, q1 = scale * acc.y;
          if (in0) dp[0] = q0;
          if (in1) dp[1] = q1;
          if constexpr (DOT) dsum += double(rv[a].x) * double(q0) + double(rv[a].y) * double(q1);
        } else {
          if (in0) dp[0] = rv[a].x - scale * acc.x;
          if (in1) dp[1] = rv[a].y - scale * acc.y;
        }
      }
    }
  }
  if constexpr (DOT) {
    // fixed-order CTA sum: warp shuffles, then the warp sums in order
    __syncthreads();  // the stages' shared memory is free
    double *red = reinterpret_cast<double *>(smem_raw);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dsum += __shfl_down_sync(0xffffffffu, dsum, o);
    if ((tid & 31) == 0) red[tid >> 5] = dsum;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
      for (int w = 0; w < NT / 32; ++w) t += red[w];
      dotp[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = t;
    }
  }
}

}  // namespace tps
