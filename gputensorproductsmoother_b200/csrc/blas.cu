// Vector kernels of the Krylov drivers.  Grid-stride loops over a fixed grid
// (kRedBlocks CTAs, a multiple of the 148 SMs), 64-bit indices, 128-bit
// vector accesses are left to the compiler for the aligned FP64 streams.
#include "blas.cuh"
#include "launch.cuh"
#include "ptx.cuh"

namespace tps {
namespace {

// entry i of a lexicographic level vector in the row-padded layout (rows of
// N1 entries sy apart); level vectors have fewer than 2^31 entries
__device__ __forceinline__ int64_t pad_index(int64_t i, PadMap pm)
{
  if (pm.sy == pm.N1) return i;
  const int row = fast_div(static_cast<int>(i), pm.m, pm.s);
  return static_cast<int64_t>(row) * pm.sy + (i - static_cast<int64_t>(row) * pm.N1);
}

// d_kind/z_kind: 0 = FP64, 1 = FP32, 2 = FP64 rounded through FP32
__device__ __forceinline__ void store_kind(void *d, int kind, int64_t i, double v)
{
  if (kind == 1)
    static_cast<float *>(d)[i] = __double2float_rn(v);
  else if (kind == 2)
    static_cast<double *>(d)[i] = static_cast<double>(__double2float_rn(v));
  else
    static_cast<double *>(d)[i] = v;
}

__device__ __forceinline__ double load_kind(const void *z, int kind, int64_t i)
{
  return kind == 1 ? static_cast<double>(static_cast<const float *>(z)[i])
                   : static_cast<const double *>(z)[i];
}

// block-wide sum of one value per thread; result valid in thread 0
template <int NT>
__device__ __forceinline__ double block_sum(double v, double *sh)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    v = l < NT / 32 ? sh[l] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  __syncthreads();
  return v;
}

__global__ void convert_d2f_kernel(float *dst, const double *src, int64_t n)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    dst[i] = __double2float_rn(src[i]);
}

__global__ void convert_f2d_kernel(double *dst, const float *src, int64_t n)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    dst[i] = static_cast<double>(src[i]);
}

__global__ void copy_d_kernel(double *dst, const double *src, int64_t n, int round32)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    dst[i] = round32 ? static_cast<double>(__double2float_rn(src[i])) : src[i];
}

template <typename T>
__global__ void copy_boundary_kernel(T *dst, const T *src, int dim, int N1)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  // one thread per boundary entry, in three coalesced groups (3D): the z = 0
  // and z = N1-1 planes, the y = 0 and y = N1-1 rows of the other planes, and
  // the x = 0 and x = N1-1 ends of the remaining rows (2D: the y rows, then
  // the x ends)
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  const int64_t n1 = N1, m = N1 - 2;
  int64_t idx;
  if (dim == 3) {
    const int64_t g0 = 2 * n1 * n1, g1 = 2 * m * n1, g2 = 2 * m * m;
    if (i < g0) {
      const int64_t f = i / (n1 * n1), r = i % (n1 * n1);
      idx = (f ? (n1 - 1) * n1 * n1 : 0) + r;
    } else if (i < g0 + g1) {
      const int64_t j = i - g0, z = 1 + j / (2 * n1), r = j % (2 * n1);
      idx = z * n1 * n1 + (r / n1 ? (n1 - 1) * n1 : 0) + r % n1;
    } else if (i < g0 + g1 + g2) {
      const int64_t j = i - g0 - g1, z = 1 + j / (2 * m), r = j % (2 * m);
      idx = z * n1 * n1 + (1 + r / 2) * n1 + (r & 1 ? n1 - 1 : 0);
    } else {
      return;
    }
  } else {
    const int64_t g0 = 2 * n1, g1 = 2 * m;
    if (i < g0) {
      idx = (i / n1 ? (n1 - 1) * n1 : 0) + i % n1;
    } else if (i < g0 + g1) {
      const int64_t j = i - g0;
      idx = (1 + j / 2) * n1 + (j & 1 ? n1 - 1 : 0);
    } else {
      return;
    }
  }
  dst[idx] = src[idx];
}

__global__ void __launch_bounds__(kRedThreads)
    dot_kernel(const double *a, const double *b, int64_t n, double *partial)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  __shared__ double sh[32];
  double s = 0.0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    s += a[i] * b[i];
  s = block_sum<kRedThreads>(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// reduce n_dots arrays of kRedBlocks partial sums; one CTA per dot
__global__ void __launch_bounds__(kRedThreads) reduce_kernel(const double *partial, double *out)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  __shared__ double sh[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < kRedBlocks; i += kRedThreads) s += partial[blockIdx.x * kRedBlocks + i];
  s = block_sum<kRedThreads>(s, sh);
  if (threadIdx.x == 0) out[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kRedThreads)
    cg_init_kernel(const double *r, const double *b, void *d, int d_kind, PadMap pm, int64_t n,
                   double *partial)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  __shared__ double sh[32];
  double s_rr = 0.0, s_bb = 0.0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double ri = r[i], bi = b[i];
    s_rr += ri * ri;
    s_bb += bi * bi;
    store_kind(d, d_kind, pad_index(i, pm), ri);
  }
  s_rr = block_sum<kRedThreads>(s_rr, sh);
  s_bb = block_sum<kRedThreads>(s_bb, sh);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = s_rr;
    partial[kRedBlocks + blockIdx.x] = s_bb;
  }
}

// sums 1..3 partial arrays sequentially in one CTA and applies `op`
template <int NDOT, typename Op>
__global__ void __launch_bounds__(kRedThreads) finalize_kernel(const double *partial, CGScalars *sc, Op op)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  __shared__ double sh[32];
  double v[NDOT];
#pragma unroll
  for (int d = 0; d < NDOT; ++d) {
    double s = 0.0;
    for (int i = threadIdx.x; i < kRedBlocks; i += kRedThreads) s += partial[d * kRedBlocks + i];
    v[d] = block_sum<kRedThreads>(s, sh);
  }
  if (threadIdx.x == 0) op(sc, v);
}

// sums `count` partial values in a fixed order in one CTA and applies `op`
template <typename Op>
__global__ void __launch_bounds__(kRedThreads) finalize_count_kernel(const double *partial, int count,
                                                                     CGScalars *sc, Op op)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  __shared__ double sh[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < count; i += kRedThreads) s += partial[i];
  double v[1] = {block_sum<kRedThreads>(s, sh)};
  if (threadIdx.x == 0) op(sc, v);
}

struct OpInit {
  __device__ void operator()(CGScalars *sc, const double *v) const
  {
    sc->rr = v[0];
    sc->bb = v[1];
    sc->breakdown = isfinite(v[0]) ? 0 : 2;
  }
};
struct OpRz {
  __device__ void operator()(CGScalars *sc, const double *v) const { sc->rz = v[0]; }
};
struct OpAlpha {
  __device__ void operator()(CGScalars *sc, const double *v) const
  {
    sc->pq = v[0];
    if (!(v[0] > 0.0) || !isfinite(v[0])) {
      sc->breakdown = isfinite(v[0]) ? 1 : 2;
      sc->alpha = 0.0;
    } else {
      sc->alpha = sc->rz / v[0];
    }
  }
};
struct OpRr {
  __device__ void operator()(CGScalars *sc, const double *v) const
  {
    sc->rr = v[0];
    if (!isfinite(v[0])) sc->breakdown = 2;
  }
};
struct OpBeta {
  __device__ void operator()(CGScalars *sc, const double *v) const
  {
    sc->zq = v[0];
    sc->rz_new = v[1];
    sc->beta = sc->rz != 0.0 ? -sc->alpha * v[0] / sc->rz : 0.0;
    sc->rz = v[1];
  }
};

__global__ void __launch_bounds__(kRedThreads)
    cg_first_direction_kernel(double *p, const void *z, int z_kind, PadMap pm, const double *r,
                              int64_t n, double *partial)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  __shared__ double sh[32];
  double s = 0.0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double zi = load_kind(z, z_kind, pad_index(i, pm));
    p[i] = zi;
    s += r[i] * zi;
  }
  s = block_sum<kRedThreads>(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kRedThreads)
    cg_update_xr_kernel(double *x, double *r, const double *p, const double *q, void *d,
                        int d_kind, PadMap pm, int64_t n, double *partial, const CGScalars *sc)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  __shared__ double sh[32];
  const double alpha = sc->alpha;
  double s = 0.0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    x[i] += alpha * p[i];
    const double ri = r[i] - alpha * q[i];
    r[i] = ri;
    s += ri * ri;
    store_kind(d, d_kind, pad_index(i, pm), ri);
  }
  s = block_sum<kRedThreads>(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kRedThreads)
    cg_dots_z_kernel(const void *z, int z_kind, PadMap pm, const double *q, const double *r,
                     int64_t n, double *partial)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  __shared__ double sh[32];
  double s1 = 0.0, s2 = 0.0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double zi = load_kind(z, z_kind, pad_index(i, pm));
    s1 += zi * q[i];
    s2 += zi * r[i];
  }
  s1 = block_sum<kRedThreads>(s1, sh);
  s2 = block_sum<kRedThreads>(s2, sh);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = s1;
    partial[kRedBlocks + blockIdx.x] = s2;
  }
}

__global__ void cg_update_p_kernel(double *p, const void *z, int z_kind, PadMap pm, int64_t n,
                                   const CGScalars *sc)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  const double beta = sc->beta;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    p[i] = load_kind(z, z_kind, pad_index(i, pm)) + beta * p[i];
}

__global__ void axpy_kernel(double *y, double a, const double *x, int64_t n)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    y[i] += a * x[i];
}

__global__ void scale_kernel(double *y, double a, int64_t n)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    y[i] *= a;
}

__global__ void sub_kernel(double *dst, const double *a, const double *b, int64_t n)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    dst[i] = a[i] - b[i];
}

__global__ void to_vcycle_kernel(void *d, int d_kind, PadMap pm, const double *src, int64_t n)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    store_kind(d, d_kind, pad_index(i, pm), src[i]);
}

__global__ void from_vcycle_kernel(double *dst, const void *z, int z_kind, PadMap pm, int64_t n)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    dst[i] = load_kind(z, z_kind, pad_index(i, pm));
}

// dense coarse solve: su[idx[i]] = sum_j inv[i][j] d[idx[j]], one warp per row
template <typename T>
__global__ void coarse_dense_kernel(const T *inv, const int *idx, int n, T *su, const T *d)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (row >= n) return;
  T s = T(0);
  for (int j = lane; j < n; j += 32) s += inv[static_cast<int64_t>(row) * n + j] * d[idx[j]];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) su[idx[row]] = s;
}

unsigned stream_grid(int64_t n, int threads)
{
  const int64_t need = (n + threads - 1) / threads;
  return static_cast<unsigned>(need < 148 * 16 ? (need > 0 ? need : 1) : 148 * 16);
}

}  // namespace

cudaError_t launch_convert_f64_to_f32(float *dst, const double *src, int64_t n, cudaStream_t s)
{
  TPS_LAUNCH((convert_d2f_kernel), stream_grid(n, 256), 256, 0, s, dst, src, n);
  return cudaGetLastError();
}
cudaError_t launch_convert_f32_to_f64(double *dst, const float *src, int64_t n, cudaStream_t s)
{
  TPS_LAUNCH((convert_f2d_kernel), stream_grid(n, 256), 256, 0, s, dst, src, n);
  return cudaGetLastError();
}
cudaError_t launch_copy_f64(double *dst, const double *src, int64_t n, int round32, cudaStream_t s)
{
  TPS_LAUNCH((copy_d_kernel), stream_grid(n, 256), 256, 0, s, dst, src, n, round32);
  return cudaGetLastError();
}
cudaError_t launch_copy_boundary(void *dst, const void *src, int dim, int N1, int elem_bytes,
                                 cudaStream_t s)
{
  const int64_t n1 = N1, m = N1 - 2;
  const int64_t count = dim == 3 ? 2 * n1 * n1 + 2 * m * n1 + 2 * m * m : 2 * n1 + 2 * m;
  const unsigned g = static_cast<unsigned>((count + 255) / 256);
  if (elem_bytes == 8)
    TPS_LAUNCH((copy_boundary_kernel<double>), g, 256, 0, s, static_cast<double *>(dst),
                                                   static_cast<const double *>(src), dim, N1);
  else
    TPS_LAUNCH((copy_boundary_kernel<float>), g, 256, 0, s, static_cast<float *>(dst),
                                                  static_cast<const float *>(src), dim, N1);
  return cudaGetLastError();
}
cudaError_t launch_dot_f64(const double *a, const double *b, int64_t n, double *partial,
                           cudaStream_t s)
{
  TPS_LAUNCH((dot_kernel), kRedBlocks, kRedThreads, 0, s, a, b, n, partial);
  return cudaGetLastError();
}
cudaError_t launch_reduce(const double *partial, int n_dots, double *out, cudaStream_t s)
{
  TPS_LAUNCH((reduce_kernel), n_dots, kRedThreads, 0, s, partial, out);
  return cudaGetLastError();
}
cudaError_t launch_cg_init(const double *r, const double *b, void *d, int d_kind, PadMap pm,
                           int64_t n, double *partial, cudaStream_t s)
{
  TPS_LAUNCH((cg_init_kernel), kRedBlocks, kRedThreads, 0, s, r, b, d, d_kind, pm, n, partial);
  return cudaGetLastError();
}
cudaError_t launch_cg_finalize_init(const double *partial, CGScalars *sc, cudaStream_t s)
{
  TPS_LAUNCH((finalize_kernel<2, OpInit>), 1, kRedThreads, 0, s, partial, sc, OpInit{});
  return cudaGetLastError();
}
cudaError_t launch_cg_first_direction(double *p, const void *z, int z_kind, PadMap pm,
                                      const double *r, int64_t n, double *partial, cudaStream_t s)
{
  TPS_LAUNCH((cg_first_direction_kernel), kRedBlocks, kRedThreads, 0, s, p, z, z_kind, pm, r, n, partial);
  return cudaGetLastError();
}
cudaError_t launch_cg_finalize_rz(const double *partial, CGScalars *sc, cudaStream_t s)
{
  TPS_LAUNCH((finalize_kernel<1, OpRz>), 1, kRedThreads, 0, s, partial, sc, OpRz{});
  return cudaGetLastError();
}
cudaError_t launch_cg_alpha_partials(const double *partial, int count, CGScalars *sc, cudaStream_t s)
{
  TPS_LAUNCH((finalize_count_kernel<OpAlpha>), 1, kRedThreads, 0, s, partial, count, sc, OpAlpha{});
  return cudaGetLastError();
}
cudaError_t launch_cg_alpha(const double *p, const double *q, int64_t n, double *partial,
                            CGScalars *sc, cudaStream_t s)
{
  TPS_LAUNCH((dot_kernel), kRedBlocks, kRedThreads, 0, s, p, q, n, partial);
  TPS_LAUNCH((finalize_kernel<1, OpAlpha>), 1, kRedThreads, 0, s, partial, sc, OpAlpha{});
  return cudaGetLastError();
}
cudaError_t launch_cg_update_xr(double *x, double *r, const double *p, const double *q, void *d,
                                int d_kind, PadMap pm, int64_t n, double *partial,
                                const CGScalars *sc, cudaStream_t s)
{
  TPS_LAUNCH((cg_update_xr_kernel), kRedBlocks, kRedThreads, 0, s, x, r, p, q, d, d_kind, pm, n, partial, sc);
  return cudaGetLastError();
}
cudaError_t launch_cg_finalize_rr(const double *partial, CGScalars *sc, cudaStream_t s)
{
  TPS_LAUNCH((finalize_kernel<1, OpRr>), 1, kRedThreads, 0, s, partial, sc, OpRr{});
  return cudaGetLastError();
}
cudaError_t launch_cg_beta(const void *z, int z_kind, PadMap pm, const double *q, const double *r,
                           int64_t n, double *partial, CGScalars *sc, cudaStream_t s)
{
  TPS_LAUNCH((cg_dots_z_kernel), kRedBlocks, kRedThreads, 0, s, z, z_kind, pm, q, r, n, partial);
  TPS_LAUNCH((finalize_kernel<2, OpBeta>), 1, kRedThreads, 0, s, partial, sc, OpBeta{});
  return cudaGetLastError();
}
cudaError_t launch_cg_update_p(double *p, const void *z, int z_kind, PadMap pm, int64_t n,
                               const CGScalars *sc, cudaStream_t s)
{
  TPS_LAUNCH((cg_update_p_kernel), stream_grid(n, 256), 256, 0, s, p, z, z_kind, pm, n, sc);
  return cudaGetLastError();
}
cudaError_t launch_axpy_f64(double *y, double a, const double *x, int64_t n, cudaStream_t s)
{
  TPS_LAUNCH((axpy_kernel), stream_grid(n, 256), 256, 0, s, y, a, x, n);
  return cudaGetLastError();
}
cudaError_t launch_scale_f64(double *y, double a, int64_t n, cudaStream_t s)
{
  TPS_LAUNCH((scale_kernel), stream_grid(n, 256), 256, 0, s, y, a, n);
  return cudaGetLastError();
}
cudaError_t launch_sub_f64(double *dst, const double *a, const double *b, int64_t n, cudaStream_t s)
{
  TPS_LAUNCH((sub_kernel), stream_grid(n, 256), 256, 0, s, dst, a, b, n);
  return cudaGetLastError();
}
cudaError_t launch_to_vcycle(void *d, int d_kind, PadMap pm, const double *src, int64_t n,
                             cudaStream_t s)
{
  TPS_LAUNCH((to_vcycle_kernel), stream_grid(n, 256), 256, 0, s, d, d_kind, pm, src, n);
  return cudaGetLastError();
}
cudaError_t launch_from_vcycle(double *dst, const void *z, int z_kind, PadMap pm, int64_t n,
                               cudaStream_t s)
{
  TPS_LAUNCH((from_vcycle_kernel), stream_grid(n, 256), 256, 0, s, dst, z, z_kind, pm, n);
  return cudaGetLastError();
}
cudaError_t launch_coarse_dense(const void *inv, const int *idx, int n_int, void *su,
                                const void *d, int elem_bytes, cudaStream_t s)
{
  const unsigned g = static_cast<unsigned>((n_int * 32 + 255) / 256);
  if (elem_bytes == 8)
    TPS_LAUNCH((coarse_dense_kernel<double>), g, 256, 0, s, static_cast<const double *>(inv), idx, n_int,
                                                  static_cast<double *>(su),
                                                  static_cast<const double *>(d));
  else
    TPS_LAUNCH((coarse_dense_kernel<float>), g, 256, 0, s, static_cast<const float *>(inv), idx, n_int,
                                                 static_cast<float *>(su),
                                                 static_cast<const float *>(d));
  return cudaGetLastError();
}

cudaError_t launch_fill(void *dst, int elem_bytes, int64_t n, cudaStream_t s)
{
  return cudaMemsetAsync(dst, 0, static_cast<size_t>(n) * elem_bytes, s);
}

namespace {

__global__ void batch_check_kernel(BatchLoop b, int first, cudaGraphConditionalHandle loop)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < b.n; i += blockDim.x) {
    const CGScalars &sc = *b.sc[i];
    if (first) {
      b.bnorm[i] = sc.bb > 0.0 ? sqrt(sc.bb) : 1.0;
      b.iters[i] = 0;
      b.active[i] = 1;
    } else if (b.active[i]) {
      b.iters[i] += 1;
    }
    if (b.active[i]) {
      const double res = sqrt(sc.rr) / b.bnorm[i];
      if (b.iters[i] < b.hist_len) b.hist[static_cast<int64_t>(i) * b.hist_len + b.iters[i]] = res;
      b.active[i] = (sc.breakdown == 0 && isfinite(res) && res > b.rel_tol && b.iters[i] < b.max_iter) ? 1 : 0;
    }
    if (b.active[i]) atomicOr(&any, 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) cudaGraphSetConditional(loop, any ? 1u : 0u);
}

__global__ void batch_select_kernel(const int *active, const __grid_constant__ BatchConds cond, int n)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  for (int i = threadIdx.x; i < n; i += blockDim.x) cudaGraphSetConditional(cond.h[i], active[i] ? 1u : 0u);
}

}  // namespace

cudaError_t launch_batch_check(BatchLoop b, int first, cudaGraphConditionalHandle loop, cudaStream_t s)
{
  TPS_LAUNCH((batch_check_kernel), 1, 256, 0, s, b, first, loop);
  return cudaGetLastError();
}

cudaError_t launch_batch_select(const int *active, const BatchConds &cond, int n, cudaStream_t s)
{
  TPS_LAUNCH((batch_select_kernel), 1, 256, 0, s, active, cond, n);
  return cudaGetLastError();
}

namespace {

// One thread waits, with the smoothers' bounded wait, on an mbarrier that
// nothing arrives on (parity 0 of a fresh barrier: its first phase never
// completes).  The wait gives up after `cycles` SM cycles and the timeout is
// recorded in `err` the way the smoother kernels record a TMA stage that did
// not arrive.
__global__ void __launch_bounds__(32) wait_timeout_selftest_kernel(int *err, long long cycles)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    if (!mbar_wait_bounded(&bar, 0, cycles)) atomicExch(err, 1);
  }
}

}  // namespace

namespace {

// n 32-bit words src -> dst (dst may be host-mapped memory)
__global__ void __launch_bounds__(32) copy_words_kernel(const uint32_t *src, uint32_t *dst, int n)
{
  griddep_wait();  // programmatic launch: the previous kernel's writes are visible
  for (int i = threadIdx.x; i < n; i += 32) dst[i] = src[i];
}

}  // namespace

cudaError_t launch_copy_words(const void *src, void *dst, int n_words, cudaStream_t s)
{
  TPS_LAUNCH((copy_words_kernel), 1, 32, 0, s, static_cast<const uint32_t *>(src), static_cast<uint32_t *>(dst),
             n_words);
  return cudaGetLastError();
}

cudaError_t launch_wait_timeout_selftest(int *err, long long cycles, cudaStream_t s)
{
  TPS_LAUNCH((wait_timeout_selftest_kernel), 1, 32, 0, s, err, cycles);
  return cudaGetLastError();
}

}  // namespace tps
