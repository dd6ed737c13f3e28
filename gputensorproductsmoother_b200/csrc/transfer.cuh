// Geometric MG transfer between a level with n_c cells per direction and its
// uniform refinement (2 n_c cells), sm_100a.
//
// Reference behaviour: MGTransferCUDA::prolongate_and_add / restrict_and_add
// (include/cuda_mg_transfer.template.cuh:575-671) with mg_kernel
// (:21-369): per coarse cell, embed the (k+1)^d coarse values into the
// (2k+1)^d child DoFs with the 1D prolongation, weight by 1/valence (0 on the
// Dirichlet boundary), atomicAdd; restriction is the transpose.  Coarse
// Dirichlet DoFs are zeroed before prolongation and after restriction.
//
// B200 design: the weighted per-cell scatter equals exact nodal interpolation
// P = P1 (x) P1 (x) P1 restricted to interior DoFs, so both directions are
// written as gathers (no atomics, deterministic):
//   fine(i)   = sum_j P1(i_z,j_z) P1(i_y,j_y) P1(i_x,j_x) coarse(j)
//   coarse(j) = sum_i P1(i_z,j_z) P1(i_y,j_y) P1(i_x,j_x) fine(i)
// A 3D transfer is one 1D pass along z plus one 2D pass per xy-plane; the
// intermediate (fine z x coarse y x coarse x, a quarter of the fine level)
// lives in a per-level scratch buffer.
#pragma once

#include "ptx.cuh"
#include "tps_common.cuh"

namespace tps {

enum class XYOut { AddInterior = 0, SetInterior = 1, SetAll = 2 };

template <int K>
struct XYTile {
  // restriction: coarse cells per CTA and direction, 8 (k <= 4) or 4, so
  // that the second pass of a 256-thread CTA has a task per thread and the
  // fine-plane halo costs (2k(C+1)+1)^2 / (2kC)^2 = 1.3x at k = 4 (1.6x with
  // 4 cells; measured at 3D Q4 64^3: FP32 85 -> 70 us, FP64 124 -> 113 us)
  static constexpr int C = K <= 4 ? 8 : 4;
  static constexpr int NT = 256;
};

// prolongation: 8 coarse cells per CTA for FP32 at k <= 4 (measured 58 -> 53
// us at 3D Q4 64^3), else 4 (k <= 4; FP64 measured 99 us with 4, 115 with 8)
// or 2
template <int K, typename T>
struct ProlTile {
  static constexpr int C = (sizeof(T) == 4 && K <= 4) ? 8 : K <= 4 ? 4 : 2;
};

// 1D prolongation of one coarse cell: v[0..k] coarse nodes -> out[0..2k-1]
// fine nodes 2k*c + f (the node 2k*(c+1) belongs to the next cell).
template <int K, typename T>
__device__ __forceinline__ void prol_cell(const T (&v)[K + 1], T (&out)[2 * K])
{
  const DegreeTables<K, T> &tb = c_tables<K, T>;
#pragma unroll
  for (int f = 0; f < 2 * K; ++f) {
    T s = T(0);
#pragma unroll
    for (int b = 0; b <= K; ++b) s += tb.prol[f * (K + 1) + b] * v[b];
    out[f] = s;
  }
}

// 1D restriction to the k coarse nodes c*k+b, b < k, from the fine nodes
// v[0..4k] = 2k(c-1) .. 2k(c+1).
template <int K, typename T>
__device__ __forceinline__ void restr_cell(const T (&v)[4 * K + 1], T (&out)[K])
{
  const DegreeTables<K, T> &tb = c_tables<K, T>;
#pragma unroll
  for (int b = 0; b < K; ++b) {
    T s = T(0);
#pragma unroll
    for (int f = 0; f <= 2 * K; ++f) s += tb.prol[f * (K + 1) + b] * v[2 * K + f];
    if (b == 0) {
      // left cell; its last child node 2k is the shared vertex counted above
#pragma unroll
      for (int f = 0; f < 2 * K; ++f) s += tb.prol[f * (K + 1) + K] * v[f];
    }
    out[b] = s;
  }
}

// ---------------------------------------------------------------------------
// xy pass, prolongation: coarse plane (N1c x N1c) -> fine plane (N1f x N1f).
// Rows are in_sy / out_sy apart; in/out advance by the plane strides per
// blockIdx.z (plane index offset by plane0).  Coarse boundary entries are read as zero when mask_in != 0.
template <int K, typename T, XYOut OUT>
__global__ void __launch_bounds__(XYTile<K>::NT)
    prolong_xy_kernel(T *__restrict__ out, const T *__restrict__ in, int N1c, int N1f,
                      int64_t in_sy, int64_t in_plane, int64_t out_sy, int64_t out_plane,
                      int plane0, int mask_in)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  constexpr int C = ProlTile<K, T>::C, NT = XYTile<K>::NT;
  constexpr int WI = C * K + 1;  // coarse inputs per direction
  constexpr int WO = 2 * K * C;  // fine outputs per direction
  __shared__ T sIn[WI * WI];
  __shared__ T sX[WI * WO];
  const int plane = plane0 + blockIdx.z;
  const T *inp = in + plane * in_plane;
  T *outp = out + plane * out_plane;
  const int cx0 = blockIdx.x * C, cy0 = blockIdx.y * C;
  // In add mode with at most one y-stage task per thread (FP64 tiles) the
  // task's current fine values are loaded first, so that the loads' latency
  // overlaps the coarse tile load and the x stage (measured at 3D Q4 64^3:
  // FP64 prolongation 0.094 -> 0.085 ms; with the two tasks of the FP32 tiles
  // the extra registers cost more than the overlap gained, 0.050 -> 0.068 ms,
  // so those tiles stage the values in shared memory instead, below)
  constexpr bool PREFETCH = OUT == XYOut::AddInterior && WO * C <= NT;
  // The other add-mode tiles (FP32) stage the current fine values of the
  // tile in shared memory by asynchronous copies, issued right after the
  // coarse tile's, so that the read-modify-write of the fine level waits on
  // no load at the end (3D Q4 64^3 mixed solve 12.35 -> 12.23 ms; the
  // coarse tile by asynchronous copies as well, 12.37 -> 12.35)
  constexpr bool STAGE_CUR = OUT == XYOut::AddInterior && !PREFETCH;
  __shared__ T sCur[STAGE_CUR ? WO * WO : 1];
  T cur[1][2 * K];
  if constexpr (PREFETCH) {
    const int t = threadIdx.x;
    const int xx = t % WO, c = t / WO;
    const int gx = 2 * K * cx0 + xx;
#pragma unroll
    for (int f = 0; f < 2 * K; ++f) {
      const int gy = 2 * K * (cy0 + c) + f;
      const bool interior = t < WO * C && gx > 0 && gx < N1f - 1 && gy > 0 && gy < N1f - 1;
      cur[0][f] = interior ? outp[gx + gy * out_sy] : T(0);
    }
  }
  {
    const uint32_t s_in = smem_u32(sIn);
    for (int e = threadIdx.x; e < WI * WI; e += NT) {
      const int lx = e % WI, ly = e / WI;
      const int gx = cx0 * K + lx, gy = cy0 * K + ly;
      const bool bnd = gx == 0 || gx == N1c - 1 || gy == 0 || gy == N1c - 1;
      const bool ok = gx < N1c && gy < N1c && !(mask_in && bnd);
      cp_async_zfill_s<sizeof(T)>(s_in + static_cast<uint32_t>(sizeof(T) * e), ok ? inp + gx + gy * in_sy : inp,
                                  ok ? static_cast<uint32_t>(sizeof(T)) : 0u);
    }
    cp_async_commit();
  }
  if constexpr (STAGE_CUR) {
    const uint32_t s_cur = smem_u32(sCur);
    for (int e = threadIdx.x; e < WO * WO; e += NT) {
      const int xx = e % WO, yy = e / WO;
      const int gx = 2 * K * cx0 + xx, gy = 2 * K * cy0 + yy;
      const bool ok = gx < N1f && gy < N1f;
      cp_async_zfill_s<sizeof(T)>(s_cur + static_cast<uint32_t>(sizeof(T) * e), ok ? outp + gx + gy * out_sy : outp,
                                  ok ? static_cast<uint32_t>(sizeof(T)) : 0u);
    }
    cp_async_commit();
    cp_async_wait_1();  // the coarse tile has landed; the fine one may be in flight
  } else {
    cp_async_wait_all();
  }
  __syncthreads();
  for (int t = threadIdx.x; t < WI * C; t += NT) {
    const int c = t % C, y = t / C;
    T v[K + 1], o[2 * K];
#pragma unroll
    for (int b = 0; b <= K; ++b) v[b] = sIn[y * WI + c * K + b];
    prol_cell<K, T>(v, o);
#pragma unroll
    for (int f = 0; f < 2 * K; ++f) sX[y * WO + c * 2 * K + f] = o[f];
  }
  if constexpr (STAGE_CUR) cp_async_wait_all();  // this thread's share of the fine tile
  __syncthreads();
  // y stage: fine rows of the tile, added to (or stored into) the fine plane
  auto y_task = [&](int t, const T (&add)[2 * K]) {
    const int xx = t % WO, c = t / WO;
    T v[K + 1], o[2 * K];
#pragma unroll
    for (int b = 0; b <= K; ++b) v[b] = sX[(c * K + b) * WO + xx];
    prol_cell<K, T>(v, o);
    const int gx = 2 * K * cx0 + xx;
    if (gx >= N1f) return;
#pragma unroll
    for (int f = 0; f < 2 * K; ++f) {
      const int gy = 2 * K * (cy0 + c) + f;
      if (gy >= N1f) continue;
      const int64_t gi = gx + gy * out_sy;
      const bool interior = gx > 0 && gx < N1f - 1 && gy > 0 && gy < N1f - 1;
      if constexpr (PREFETCH) {
        if (interior) outp[gi] = add[f] + o[f];
      } else if constexpr (STAGE_CUR) {
        if (interior) outp[gi] = sCur[(2 * K * c + f) * WO + xx] + o[f];
      } else if constexpr (OUT == XYOut::AddInterior) {
        if (interior) outp[gi] += o[f];
      } else if constexpr (OUT == XYOut::SetInterior) {
        if (interior) outp[gi] = o[f];
      } else {
        outp[gi] = o[f];
      }
    }
  };
  if constexpr (PREFETCH) {
    if (threadIdx.x < WO * C) y_task(threadIdx.x, cur[0]);
  } else {
    for (int t = threadIdx.x; t < WO * C; t += NT) y_task(t, cur[0]);
  }
}

// xy pass, restriction: fine plane -> coarse plane.  Fine boundary entries
// are read as zero (weight 0 on Dirichlet DoFs).  zero_plane != 0 writes
// zeros instead (fine z-boundary planes).
template <int K, typename T, XYOut OUT>
__global__ void __launch_bounds__(XYTile<K>::NT)
    restrict_xy_kernel(T *__restrict__ out, const T *__restrict__ in, int N1c, int N1f,
                       int64_t in_sy, int64_t in_plane, int64_t out_sy, int64_t out_plane,
                       int plane0, int n_planes_total)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  constexpr int C = XYTile<K>::C, NT = XYTile<K>::NT;
  constexpr int WI = 2 * K * (C + 1) + 1;  // fine inputs per direction
  constexpr int WO = C * K;                // coarse outputs per direction
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T *sIn = reinterpret_cast<T *>(smem_raw);
  T *sX = sIn + WI * WI;
  const int plane = plane0 + blockIdx.z;
  const bool zero_plane = n_planes_total > 1 && (plane == 0 || plane == n_planes_total - 1);
  const T *inp = in + plane * in_plane;
  T *outp = out + plane * out_plane;
  const int cx0 = blockIdx.x * C, cy0 = blockIdx.y * C;
  const int fx0 = 2 * K * (cx0 - 1), fy0 = 2 * K * (cy0 - 1);
  // the fine tile (with its halo) by asynchronous copies, all in flight at
  // once; a loop of plain loads waited on each (measured at 3D 64^3, us per
  // restriction, plain / asynchronous: Q4 FP32 69.9 / 56.9, Q4 FP64 112.8 /
  // 92.3, Q3 FP64 37.7 / 33.1; Q7 32^3 FP64 101.5 / 65.9, FP32 51.3 / 56.0);
  // entries outside the interior are zero-filled
  const uint32_t s_in = smem_u32(sIn);
  for (int e = threadIdx.x; e < WI * WI; e += NT) {
    const int lx = e % WI, ly = e / WI;
    const int gx = fx0 + lx, gy = fy0 + ly;
    const bool ok = !zero_plane && gx > 0 && gx < N1f - 1 && gy > 0 && gy < N1f - 1;
    cp_async_zfill_s<sizeof(T)>(s_in + static_cast<uint32_t>(sizeof(T) * e), ok ? inp + gx + gy * in_sy : inp,
                                ok ? static_cast<uint32_t>(sizeof(T)) : 0u);
  }
  cp_async_commit();
  cp_async_wait_all();
  __syncthreads();
  for (int t = threadIdx.x; t < WI * C; t += NT) {
    const int c = t % C, y = t / C;
    T v[4 * K + 1], o[K];
#pragma unroll
    for (int j = 0; j <= 4 * K; ++j) v[j] = sIn[y * WI + c * 2 * K + j];
    restr_cell<K, T>(v, o);
#pragma unroll
    for (int b = 0; b < K; ++b) sX[y * WO + c * K + b] = o[b];
  }
  __syncthreads();
  for (int t = threadIdx.x; t < WO * C; t += NT) {
    const int xx = t % WO, c = t / WO;
    T v[4 * K + 1], o[K];
#pragma unroll
    for (int j = 0; j <= 4 * K; ++j) v[j] = sX[(c * 2 * K + j) * WO + xx];
    restr_cell<K, T>(v, o);
    const int gx = K * cx0 + xx;
    if (gx >= N1c) continue;
#pragma unroll
    for (int b = 0; b < K; ++b) {
      const int gy = K * (cy0 + c) + b;
      if (gy >= N1c) continue;
      const int64_t gi = gx + gy * out_sy;
      const bool interior = gx > 0 && gx < N1c - 1 && gy > 0 && gy < N1c - 1;
      if constexpr (OUT == XYOut::AddInterior) {
        if (interior) outp[gi] += o[b];
      } else if constexpr (OUT == XYOut::SetInterior) {
        if (interior) outp[gi] = o[b];
      } else {
        outp[gi] = o[b];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// z pass, prolongation: coarse (N1c planes of P entries) -> tmp (N1f planes of
// P entries), P = N1c^2.  Input entries on the coarse boundary read as zero
// (MASK) or as they are (the FMG prolongation of the solution).
template <int K, typename T, bool MASK = true>
__global__ void prolong_z_kernel(T *__restrict__ tmp, const T *__restrict__ coarse, int N1c,
                                 int N1f, int n_cells_c, int64_t c_sy, int64_t c_sz)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  const int64_t P = static_cast<int64_t>(N1c) * N1c;
  const int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  const int c = blockIdx.y;  // coarse cell along z
  if (idx >= P) return;
  const int gy = static_cast<int>(idx) / N1c, gx = static_cast<int>(idx) - gy * N1c;  // idx < N1c^2 < 2^31
  const bool bxy = gx == 0 || gx == N1c - 1 || gy == 0 || gy == N1c - 1;
  T v[K + 1], o[2 * K];
#pragma unroll
  for (int b = 0; b <= K; ++b) {
    const int gz = c * K + b;
    v[b] = (MASK && (bxy || gz == 0 || gz == N1c - 1)) ? T(0) : __ldg(&coarse[gz * c_sz + gy * c_sy + gx]);
  }
  prol_cell<K, T>(v, o);
#pragma unroll
  for (int f = 0; f < 2 * K; ++f) tmp[(2 * K * c + f) * P + idx] = o[f];
  if (c == n_cells_c - 1) tmp[(N1f - 1) * P + idx] = MASK ? T(0) : v[K];
}

// z pass, restriction: tmp (N1f planes of P = N1c^2 entries) -> coarse.
template <int K, typename T, bool ADD>
__global__ void restrict_z_kernel(T *__restrict__ coarse, const T *__restrict__ tmp, int N1c,
                                  int N1f, int64_t c_sy, int64_t c_sz)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  const int64_t P = static_cast<int64_t>(N1c) * N1c;
  const int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  const int c = blockIdx.y;  // coarse cell along z: outputs c*k + b, b < k
  if (idx >= P) return;
  const int gy = static_cast<int>(idx) / N1c, gx = static_cast<int>(idx) - gy * N1c;  // idx < N1c^2 < 2^31
  if (gx == 0 || gx == N1c - 1 || gy == 0 || gy == N1c - 1) return;
  T v[4 * K + 1], o[K];
#pragma unroll
  for (int j = 0; j <= 4 * K; ++j) {
    const int fz = 2 * K * (c - 1) + j;
    v[j] = (fz <= 0 || fz >= N1f - 1) ? T(0) : __ldg(&tmp[fz * P + idx]);
  }
  restr_cell<K, T>(v, o);
#pragma unroll
  for (int b = 0; b < K; ++b) {
    const int gz = c * K + b;
    if (gz == 0 || gz >= N1c - 1) continue;
    T &dst = coarse[gz * c_sz + gy * c_sy + gx];
    if constexpr (ADD)
      dst += o[b];
    else
      dst = o[b];
  }
}

}  // namespace tps
