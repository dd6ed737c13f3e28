// Variable-coefficient (-div(kappa grad u), kappa constant per cell) kernels
// and the adjoint helpers.  No reference counterpart: the reference's Poisson
// path has a unit coefficient (include/laplace_operator.cuh:25-31); these
// kernels extend the same Q_k discretisation with a per-cell factor.
//
//  * cell_apply_kernel: y += sum over the cells of ONE colour (cell index
//    parities) of kappa_c * A_cell x_c.  Cells of one colour share no DoF, so
//    the read-modify-write needs no atomics; 2^d launches give A(kappa) x in a
//    fixed order (deterministic).
//  * kappa_smoother_kernel: one patch per CTA, box residual b - A(kappa) x
//    assembled cell by cell (the patch's 2^d cells), local solve by fast
//    diagonalization of the unit-coefficient patch scaled by the
//    patch-averaged coefficient per DoF, D^-1/2 FD^-1 D^-1/2 with D_i the
//    mean kappa of the patch cells containing DoF i (exact on couplings
//    inside one cell; one scalar mean per patch stagnates for strongly
//    varying kappa),
//    x_I <- x_I + omega * delta (the residual form is kept because the
//    approximate local solve does not cancel x_I).
//  * cell_energy_kernel: e_c = lambda_c^T (A_cell u_c) = int_c grad(lambda).grad(u)
//    for dJ/dkappa_c = -e_c.
#pragma once

#include "tps_common.cuh"

namespace tps {

// local stiffness product of one cell held in shared memory (n = k+1 nodes
// per direction): out = s * sum_d (L in direction d, M elsewhere) in.
// Lines are distributed over `nthreads` threads starting at `t0`.
template <int DIM, int K, typename T>
__device__ __forceinline__ void cell_local_apply(const T *in, T *out, T *t1, T *t2, T s, int t0,
                                                 int nthreads)
{
  constexpr int NP = K + 1;
  constexpr int LINES = DIM == 3 ? NP * NP : NP;
  const DegreeTables<K, T> &tb = c_tables<K, T>;
  // x
  for (int l = t0; l < LINES; l += nthreads) {
    T v[NP];
#pragma unroll
    for (int j = 0; j < NP; ++j) v[j] = in[l * NP + j];
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      T a = T(0), c = T(0);
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        a += tb.cmass[i * NP + j] * v[j];
        c += tb.clap[i * NP + j] * v[j];
      }
      t1[l * NP + i] = a;
      t2[l * NP + i] = c;
    }
  }
  __syncthreads();
  if constexpr (DIM == 2) {
    for (int xx = t0; xx < NP; xx += nthreads) {
      T a[NP], c[NP];
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        a[j] = t1[j * NP + xx];
        c[j] = t2[j * NP + xx];
      }
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        T acc = T(0);
#pragma unroll
        for (int j = 0; j < NP; ++j) acc += tb.clap[i * NP + j] * a[j] + tb.cmass[i * NP + j] * c[j];
        out[i * NP + xx] = s * acc;
      }
    }
  } else {
    // y: u1 = M t1 -> in-place into a scratch? use out as u1 and in-place t2 update
    // u1 = M_y t1 (stored in out), u2 = L_y t1 + M_y t2 (stored in t1 after use)
    for (int l = t0; l < NP * NP; l += nthreads) {
      const int z = l / NP, xx = l % NP;
      T a[NP], c[NP];
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        a[j] = t1[(z * NP + j) * NP + xx];
        c[j] = t2[(z * NP + j) * NP + xx];
      }
      T u1[NP], u2[NP];
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        T p = T(0), q = T(0);
#pragma unroll
        for (int j = 0; j < NP; ++j) {
          p += tb.cmass[i * NP + j] * a[j];
          q += tb.clap[i * NP + j] * a[j] + tb.cmass[i * NP + j] * c[j];
        }
        u1[i] = p;
        u2[i] = q;
      }
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        out[(z * NP + i) * NP + xx] = u1[i];
        t2[(z * NP + i) * NP + xx] = u2[i];
      }
    }
    __syncthreads();
    // z: out = s (L_z u1 + M_z u2)
    for (int l = t0; l < NP * NP; l += nthreads) {
      T a[NP], c[NP];
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        a[j] = out[j * NP * NP + l];
        c[j] = t2[j * NP * NP + l];
      }
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        T acc = T(0);
#pragma unroll
        for (int j = 0; j < NP; ++j) acc += tb.clap[i * NP + j] * a[j] + tb.cmass[i * NP + j] * c[j];
        t1[i * NP * NP + l] = s * acc;
      }
    }
    __syncthreads();
    for (int l = t0; l < NP * NP * NP; l += nthreads) out[l] = t1[l];
  }
  __syncthreads();
}

template <int DIM, int K>
struct KappaCfg {
  static constexpr int NP = K + 1;
  static constexpr int CELL = DIM == 3 ? NP * NP * NP : NP * NP;
  static constexpr int NT = 128;
};

// local mass product of one cell: out = s * (M (x) ... (x) M) in
template <int DIM, int K, typename T>
__device__ __forceinline__ void cell_local_mass(const T *in, T *out, T *t1, T s, int t0, int nthreads)
{
  constexpr int NP = K + 1;
  const DegreeTables<K, T> &tb = c_tables<K, T>;
  constexpr int CELL = DIM == 3 ? NP * NP * NP : NP * NP;
  const T *src = in;
  T *bufs[2] = {out, t1};
  for (int dir = 0; dir < DIM; ++dir) {
    T *dstb = bufs[(DIM - 1 - dir) & 1];  // alternate so the last direction lands in `out`
    const int stride = dir == 0 ? 1 : dir == 1 ? NP : NP * NP;
    for (int l = t0; l < CELL / NP; l += nthreads) {
      int bidx;
      if (dir == 0) bidx = l * NP;
      else if (dir == 1) bidx = (l / NP) * NP * NP + l % NP;
      else bidx = l;
      T v[NP];
#pragma unroll
      for (int j = 0; j < NP; ++j) v[j] = src[bidx + j * stride];
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        T acc = T(0);
#pragma unroll
        for (int j = 0; j < NP; ++j) acc += tb.cmass[i * NP + j] * v[j];
        dstb[bidx + i * stride] = dir == DIM - 1 ? s * acc : acc;
      }
    }
    __syncthreads();
    src = dstb;
  }
}

// dst += kappa_c * s * A_cell src_c (or s * M_cell src_c when MASS) for the
// cells of colour `colour` (one cell per CTA; cells of one colour are two
// apart, so no conflicts)
template <int DIM, int K, typename T, bool MASS>
__global__ void __launch_bounds__(KappaCfg<DIM, K>::NT)
    cell_apply_kernel(T *__restrict__ dst, const T *__restrict__ src, const T *__restrict__ kappa,
                      int n, int colour, int ncx, int ncy, int64_t sy, int64_t sz, T s)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  using C = KappaCfg<DIM, K>;
  constexpr int NP = C::NP;
  __shared__ T in[C::CELL], out[C::CELL], t1[C::CELL], t2[C::CELL];
  const int j = blockIdx.x;
  const int px = colour & 1, py = (colour >> 1) & 1, pz = (colour >> 2) & 1;
  const int cx = px + 2 * (j % ncx), cy = py + 2 * ((j / ncx) % ncy);
  const int cz = DIM == 3 ? pz + 2 * (j / (ncx * ncy)) : 0;
  const int64_t base = int64_t(cx) * K + int64_t(cy) * K * sy + int64_t(cz) * K * sz;
  for (int l = threadIdx.x; l < C::CELL; l += C::NT) {
    const int lx = l % NP, ly = (l / NP) % NP, lz = DIM == 3 ? l / (NP * NP) : 0;
    in[l] = src[base + lx + ly * sy + lz * sz];
  }
  __syncthreads();
  const int64_t cidx = int64_t(cx) + int64_t(cy) * n + (DIM == 3 ? int64_t(cz) * n * n : 0);
  if constexpr (MASS)
    cell_local_mass<DIM, K, T>(in, out, t1, s, threadIdx.x, C::NT);
  else
    cell_local_apply<DIM, K, T>(in, out, t1, t2, s * kappa[cidx], threadIdx.x, C::NT);
  for (int l = threadIdx.x; l < C::CELL; l += C::NT) {
    const int lx = l % NP, ly = (l / NP) % NP, lz = DIM == 3 ? l / (NP * NP) : 0;
    dst[base + lx + ly * sy + lz * sz] += out[l];
  }
}

// finishing pass of the cell-accumulated operator: Dirichlet rows set to 0
// (they received cell contributions), and with a right-hand side the
// interior rows become the residual rhs - dst
template <int DIM, typename T>
__global__ void finish_residual_kernel(T *__restrict__ dst, const T *__restrict__ rhs, int N1,
                                       int64_t sy, int64_t sz)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  const int64_t rows = DIM == 3 ? int64_t(N1) * N1 : N1;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < rows * N1;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int x = int(i % N1);
    const int64_t r = i / N1;
    const int y = int(r % N1), z = DIM == 3 ? int(r / N1) : 0;
    const int64_t gi = x + y * sy + z * sz;
    const bool bnd = x == 0 || x == N1 - 1 || y == 0 || y == N1 - 1 ||
                     (DIM == 3 && (z == 0 || z == N1 - 1));
    if (bnd)
      dst[gi] = T(0);
    else if (rhs)
      dst[gi] = rhs[gi] - dst[gi];
  }
}

// e_c = lambda_c^T (s A_cell u_c) for every cell (FP64)
template <int DIM, int K>
__global__ void __launch_bounds__(KappaCfg<DIM, K>::NT)
    cell_energy_kernel(double *__restrict__ e, const double *__restrict__ u,
                       const double *__restrict__ lam, int n, int64_t sy, int64_t sz, double s)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  using C = KappaCfg<DIM, K>;
  constexpr int NP = C::NP;
  __shared__ double in[C::CELL], out[C::CELL], t1[C::CELL], t2[C::CELL];
  __shared__ double red[C::NT / 32];
  const int64_t c = blockIdx.x;
  const int cx = int(c % n), cy = int((c / n) % n), cz = DIM == 3 ? int(c / (int64_t(n) * n)) : 0;
  const int64_t base = int64_t(cx) * K + int64_t(cy) * K * sy + int64_t(cz) * K * sz;
  for (int l = threadIdx.x; l < C::CELL; l += C::NT) {
    const int lx = l % NP, ly = (l / NP) % NP, lz = DIM == 3 ? l / (NP * NP) : 0;
    in[l] = u[base + lx + ly * sy + lz * sz];
  }
  __syncthreads();
  cell_local_apply<DIM, K, double>(in, out, t1, t2, s, threadIdx.x, C::NT);
  double acc = 0.0;
  for (int l = threadIdx.x; l < C::CELL; l += C::NT) {
    const int lx = l % NP, ly = (l / NP) % NP, lz = DIM == 3 ? l / (NP * NP) : 0;
    acc += lam[base + lx + ly * sy + lz * sz] * out[l];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < C::NT / 32; ++w) t += red[w];
    e[c] = t;
  }
}

// kappa smoother: one patch of colour `colour` per CTA
template <int DIM, int K, typename T>
struct KSm {
  static constexpr int NP = K + 1, N1 = 2 * K + 1, M = 2 * K - 1;
  static constexpr int NC = 1 << DIM;  // cells of a patch
  static constexpr int BOX = DIM == 3 ? N1 * N1 * N1 : N1 * N1;
  static constexpr int INT = DIM == 3 ? M * M * M : M * M;
  static constexpr int CELL = DIM == 3 ? NP * NP * NP : NP * NP;
  static constexpr int NT = DIM == 3 ? 256 : 128;
  // X[BOX] | TA | TB | UA | UB (NC cells each); the local solve reuses UA, UB
  static constexpr int ELEMS = BOX + 4 * NC * CELL;
  static_assert(NC * CELL >= INT, "the local-solve buffers live in the cell buffers");
};

// kappa patch smoother: one CTA per patch.  The box residual is assembled
// from the 2^d cells of the patch contracted at once (each 1D stage has a
// line task per cell and line, so the CTA's threads share all cells' work),
// the per-cell results are combined per interior node, then the local solve.
template <int DIM, int K, typename T>
__global__ void __launch_bounds__(KSm<DIM, K, T>::NT)
    kappa_smoother_kernel(T *__restrict__ x, const T *__restrict__ b, const T *__restrict__ kappa,
                          int n, int colour, int nx_c, int ny_c, int64_t sy, int64_t sz, T s,
                          T fd_scale, T omega)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  using S = KSm<DIM, K, T>;
  constexpr int NP = S::NP, N1 = S::N1, M = S::M, NT = S::NT, NC = S::NC, CELL = S::CELL;
  const DegreeTables<K, T> &tb = c_tables<K, T>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ T kps[NC];  // the patch cells' coefficients (indexed by run-time cell)
  T *X = reinterpret_cast<T *>(smem_raw);
  T *TA = X + S::BOX, *TB = TA + NC * CELL, *UA = TB + NC * CELL, *UB = UA + NC * CELL;
  T *Q1 = UA, *Q2 = UB;  // local solve, after the residual is assembled
  const int j = blockIdx.x;
  const int px = (colour & 1) + 2 * (j % nx_c);
  const int py = ((colour >> 1) & 1) + 2 * (DIM == 3 ? (j / nx_c) % ny_c : j / nx_c);
  const int pz = DIM == 3 ? ((colour >> 2) & 1) + 2 * (j / (nx_c * ny_c)) : 0;
  const int64_t first = int64_t(px) * K + int64_t(py) * K * sy + int64_t(pz) * K * sz;
  for (int l = threadIdx.x; l < S::BOX; l += NT) {
    const int lx = l % N1, ly = (l / N1) % N1, lz = DIM == 3 ? l / (N1 * N1) : 0;
    X[l] = x[first + lx + ly * sy + lz * sz];
  }
  T kpat[NC];
#pragma unroll
  for (int cc = 0; cc < NC; ++cc) {
    const int ox = cc & 1, oy = (cc >> 1) & 1, oz = (cc >> 2) & 1;
    kpat[cc] = kappa[int64_t(px + ox) + int64_t(py + oy) * n + (DIM == 3 ? int64_t(pz + oz) * n * n : 0)];
  }
  if (threadIdx.x < NC) {
#pragma unroll
    for (int cc = 0; cc < NC; ++cc)
      if (cc == threadIdx.x) kps[cc] = kpat[cc];
  }
  __syncthreads();
  constexpr int LINES = CELL / NP;  // lines of one cell along one direction
  // x: TA = M_x x_c, TB = L_x x_c, per cell [c][z][y][x]
  for (int t = threadIdx.x; t < NC * LINES; t += NT) {
    const int cc = t / LINES, r = t % LINES;
    const int ox = cc & 1, oy = (cc >> 1) & 1, oz = (cc >> 2) & 1;
    const int yl = r % NP, zl = DIM == 3 ? r / NP : 0;
    const T *src = X + (DIM == 3 ? (oz * K + zl) * N1 * N1 : 0) + (oy * K + yl) * N1 + ox * K;
    T v[NP];
#pragma unroll
    for (int q = 0; q < NP; ++q) v[q] = src[q];
    T *da = TA + cc * CELL + r * NP, *db = TB + cc * CELL + r * NP;
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      T a = T(0), c = T(0);
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        a += tb.cmass[i * NP + q] * v[q];
        c += tb.clap[i * NP + q] * v[q];
      }
      da[i] = a;
      db[i] = c;
    }
  }
  __syncthreads();
  if constexpr (DIM == 3) {
    // y: UA = M_y TA, UB = L_y TA + M_y TB
    for (int t = threadIdx.x; t < NC * LINES; t += NT) {
      const int cc = t / LINES, r = t % LINES;
      const int xl = r % NP, zl = r / NP;
      const T *sa = TA + cc * CELL + zl * NP * NP + xl, *sb = TB + cc * CELL + zl * NP * NP + xl;
      T va[NP], vb[NP];
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        va[q] = sa[q * NP];
        vb[q] = sb[q * NP];
      }
      T *da = UA + cc * CELL + zl * NP * NP + xl, *db = UB + cc * CELL + zl * NP * NP + xl;
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        T a = T(0), c = T(0);
#pragma unroll
        for (int q = 0; q < NP; ++q) {
          a += tb.cmass[i * NP + q] * va[q];
          c += tb.clap[i * NP + q] * va[q] + tb.cmass[i * NP + q] * vb[q];
        }
        da[i * NP] = a;
        db[i * NP] = c;
      }
    }
    __syncthreads();
    // z: TA = s kappa_c (L_z UA + M_z UB) = the cell's A_c x_c
    for (int t = threadIdx.x; t < NC * LINES; t += NT) {
      const int cc = t / LINES, r = t % LINES;
      const T *sa = UA + cc * CELL + r, *sb = UB + cc * CELL + r;
      T va[NP], vb[NP];
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        va[q] = sa[q * NP * NP];
        vb[q] = sb[q * NP * NP];
      }
      const T sk = s * kps[cc];
      T *d = TA + cc * CELL + r;
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        T a = T(0);
#pragma unroll
        for (int q = 0; q < NP; ++q) a += tb.clap[i * NP + q] * va[q] + tb.cmass[i * NP + q] * vb[q];
        d[i * NP * NP] = sk * a;
      }
    }
  } else {
    // y: UA = s kappa_c (L_y TA + M_y TB)
    for (int t = threadIdx.x; t < NC * LINES; t += NT) {
      const int cc = t / LINES, xl = t % LINES;
      const T *sa = TA + cc * CELL + xl, *sb = TB + cc * CELL + xl;
      T va[NP], vb[NP];
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        va[q] = sa[q * NP];
        vb[q] = sb[q * NP];
      }
      const T sk = s * kps[cc];
      T *d = UA + cc * CELL + xl;
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        T a = T(0);
#pragma unroll
        for (int q = 0; q < NP; ++q) a += tb.clap[i * NP + q] * va[q] + tb.cmass[i * NP + q] * vb[q];
        d[i * NP] = sk * a;
      }
    }
  }
  __syncthreads();
  const T *OUT = DIM == 3 ? TA : UA;
  // D^-1/2 of interior DoF l: mean kappa of the patch cells containing it
  auto dinv_sqrt = [&](int l) -> T {
    const int c3[3] = {l % M + 1, (l / M) % M + 1, DIM == 3 ? l / (M * M) + 1 : 0};
    T acc = T(0);
    int cnt = 0;
#pragma unroll
    for (int cc = 0; cc < NC; ++cc) {
      bool in = true;
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        const int o = (cc >> d) & 1;
        in = in && !(o == 0 && c3[d] > K) && !(o == 1 && c3[d] < K);
      }
      if (in) {
        acc += kpat[cc];
        ++cnt;
      }
    }
    return T(1) / sqrt(acc / T(cnt));
  };
  // (A(kappa) x)_l of interior node l: the sum over the patch cells containing it
  auto ax_node = [&](int l) -> T {
    const int c3[3] = {l % M + 1, (l / M) % M + 1, DIM == 3 ? l / (M * M) + 1 : 0};
    T acc = T(0);
#pragma unroll
    for (int cc = 0; cc < NC; ++cc) {
      bool in = true;
      int li = 0, mul = 1;
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        const int o = (cc >> d) & 1;
        in = in && !(o == 0 && c3[d] > K) && !(o == 1 && c3[d] < K);
        li += (c3[d] - o * K) * mul;
        mul *= NP;
      }
      if (in) acc += OUT[cc * CELL + li];
    }
    return acc;
  };
  // interior residual r = D^-1/2 (b_I - (A(kappa) x)_I); Q1 overlaps the cell
  // results in 2D, so all of them are combined before Q1 is written
  constexpr int RU = (S::INT + NT - 1) / NT;
  T rloc[RU];
#pragma unroll
  for (int u = 0; u < RU; ++u) {
    const int l = threadIdx.x + u * NT;
    if (l < S::INT) {
      const int lx = l % M + 1, ly = (l / M) % M + 1, lz = DIM == 3 ? l / (M * M) + 1 : 0;
      rloc[u] = (b[first + lx + ly * sy + lz * sz] - ax_node(l)) * dinv_sqrt(l);
    }
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < RU; ++u) {
    const int l = threadIdx.x + u * NT;
    if (l < S::INT) Q1[l] = rloc[u];
  }
  __syncthreads();
  // fast diagonalization: S^T along each direction, scale, S back (ping-pong Q1/Q2)
  T *src = Q1, *dst = Q2;
  for (int pass = 0; pass < 2 * DIM; ++pass) {
    const int dir = pass % DIM;
    const bool tr = pass < DIM;
    const int stride = dir == 0 ? 1 : dir == 1 ? M : M * M;
    const int lines = S::INT / M;
    for (int l = threadIdx.x; l < lines; l += NT) {
      // base index of line l along dir
      int bidx;
      if (dir == 0) bidx = l * M;
      else if (dir == 1) bidx = (l / M) * M * M + l % M;
      else bidx = l;
      T v[M], q[M];
#pragma unroll
      for (int i = 0; i < M; ++i) v[i] = src[bidx + i * stride];
#pragma unroll
      for (int i = 0; i < M; ++i) {
        T acc = T(0);
#pragma unroll
        for (int jj = 0; jj < M; ++jj)
          acc += (tr ? tb.evec[jj * M + i] : tb.evec[i * M + jj]) * v[jj];
        q[i] = acc;
      }
      if (pass == DIM - 1) {
        // divide by the eigenvalue sums (modes), scaled back to physical cells
#pragma unroll
        for (int i = 0; i < M; ++i) {
          const int e = bidx + i * stride;
          const int mx = e % M, my = (e / M) % M, mz = DIM == 3 ? e / (M * M) : 0;
          const T lam = tb.eval[mx] + tb.eval[my] + (DIM == 3 ? tb.eval[mz] : T(0));
          q[i] = q[i] * fd_scale / lam;
        }
      }
#pragma unroll
      for (int i = 0; i < M; ++i) dst[bidx + i * stride] = q[i];
    }
    __syncthreads();
    T *tmp = src;
    src = dst;
    dst = tmp;
  }
  for (int l = threadIdx.x; l < S::INT; l += NT) {
    const int lx = l % M + 1, ly = (l / M) % M + 1, lz = DIM == 3 ? l / (M * M) + 1 : 0;
    x[first + lx + ly * sy + lz * sz] = omega * (X[lx + ly * N1 + lz * N1 * N1] + src[l] * dinv_sqrt(l));
  }
}

}  // namespace tps
