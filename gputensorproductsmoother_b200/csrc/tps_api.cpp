// C-ABI implementation: problem set-up, level operators, the V-cycle and the
// FP64 Krylov drivers (host C++, CUDA runtime only; no torch, no deal.II).
//
// Reference counterparts:
//   tps_create        MultigridSolvers ctor (include/solver.cuh:1545-1744),
//                     LevelVertexPatch::reinit (include/patch_base.template.cuh:194-307),
//                     MGTransferCUDA::build (include/cuda_mg_transfer.template.cuh:453-559)
//   tps_laplace_vmult LaplaceOperator::vmult (include/laplace_operator.cuh:86-101)
//   tps_smoother_step PatchSmootherImpl::vmult/step (include/patch_smoother.cuh:155-292)
//   tps_prolongate_add / tps_restrict_add
//                     MGTransferCUDA (include/cuda_mg_transfer.template.cuh:575-671)
//   tps_vcycle        MultigridSolvers::vmult + v_cycle (include/solver.cuh:1915-2001)
//   tps_solve         MultigridSolvers::solve_gmres (include/solver.cuh:1865-1910) and the
//                     MG-preconditioned flexible CG driver (no reference counterpart)
#include "../../include/tps.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "blas.cuh"
#include "fe_data.h"
#include "kernel_table.h"

// NVTX ranges around the solver phases (header-only NVTX v3; without an
// attached tool each range is a check of one function pointer).  Ranges in
// code that is captured into a CUDA graph mark the capture, not its replays.
#ifndef TPS_NVTX
#define TPS_NVTX 1
#endif
#if TPS_NVTX
#include <nvtx3/nvToolsExt.h>
namespace tps {
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};
}  // namespace tps
#define TPS_RANGE_CAT_(a, b) a##b
#define TPS_RANGE_CAT(a, b) TPS_RANGE_CAT_(a, b)
#define TPS_RANGE(name) ::tps::NvtxRange TPS_RANGE_CAT(tps_nvtx_, __LINE__)(name)
#else
#define TPS_RANGE(name) ((void)0)
#endif

namespace tps {

const KernelTable *kernel_table(int degree)
{
  switch (degree) {
    case 1: return &kernel_table_k1;
    case 2: return &kernel_table_k2;
    case 3: return &kernel_table_k3;
    case 4: return &kernel_table_k4;
    case 5: return &kernel_table_k5;
    case 6: return &kernel_table_k6;
    case 7: return &kernel_table_k7;
    default: return nullptr;
  }
}

// coarse dense solve kernels (FP64 inverse rounded to the V-cycle precision)
cudaError_t launch_coarse_dense(const void *inv, const int *idx, int n_int, void *su,
                                const void *d, int elem_bytes, cudaStream_t s);

}  // namespace tps

using namespace tps;

namespace {
thread_local std::string g_create_error;
}  // namespace

namespace tps {
void set_handle_free_error(const std::string &msg) { g_create_error = msg; }
}  // namespace tps

namespace {

struct ApiError : std::runtime_error {
  int code;
  ApiError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define TPS_CUDA(call)                                                                       \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      throw ApiError(e_ == cudaErrorMemoryAllocation ? TPS_ERR_ALLOC : TPS_ERR_CUDA,         \
                     std::string(#call) + ": " + cudaGetErrorString(e_));                    \
  } while (0)

// tps_inject_alloc_failure: the n-th device allocation from now fails; 0 = off
std::atomic<int> g_alloc_fault{0};

bool injected_alloc_fault()
{
  int n = g_alloc_fault.load();
  while (n > 0)
    if (g_alloc_fault.compare_exchange_weak(n, n - 1)) return n == 1;
  return false;
}

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { release(); }
  void release()
  {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  void alloc(size_t b)
  {
    release();
    if (b == 0) return;
    if (injected_alloc_fault())
      throw ApiError(TPS_ERR_ALLOC, "cudaMalloc: out of memory (injected by tps_inject_alloc_failure)");
    cudaError_t e = cudaMalloc(&p, b);
    if (e != cudaSuccess) {
      p = nullptr;
      throw ApiError(TPS_ERR_ALLOC, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    bytes = b;
    TPS_CUDA(cudaMemset(p, 0, b));
  }
  template <typename T>
  T *as() const { return static_cast<T *>(p); }
};

// A small host-mapped pinned buffer: kernels write scalars there, the host
// reads them after synchronizing the stream.
struct Mailbox {
  void *host = nullptr;
  Mailbox() = default;
  Mailbox(const Mailbox &) = delete;
  Mailbox &operator=(const Mailbox &) = delete;
  ~Mailbox()
  {
    if (host) cudaFreeHost(host);
  }
  static constexpr size_t kBytes = 256;
  void ensure()
  {
    if (host) return;
    cudaError_t e = cudaHostAlloc(&host, kBytes, cudaHostAllocMapped);
    if (e != cudaSuccess) {
      host = nullptr;
      throw ApiError(TPS_ERR_ALLOC, std::string("cudaHostAlloc: ") + cudaGetErrorString(e));
    }
  }
};

// V-cycle work vectors of one precision.  In 3D their rows are padded to a
// 16-byte pitch so the smoother can stage patch boxes with TMA.
struct VcycleVectors {
  bool ready = false;
  std::vector<std::unique_ptr<DevBuf>> d, su, t, tmp;  // per level
  std::vector<VecLayout> layout;                       // per level
  std::vector<SmootherMaps> maps;                      // TMA descriptors (x = su, b = d)
  DevBuf coarse_inv;                                   // dense coarse inverse
  DevBuf coarse_idx;                                   // interior DoFs of the coarse level
};

}  // namespace

struct tps_handle {
  int dim = 0, k = 0, n_coarse = 0, n_levels = 0, device = 0;
  int n_sm = 148;  // multiprocessors of the device
  double omega = 1.0;
  std::vector<LevelGeomH> lv;
  const KernelTable *kt = nullptr;
  DegreeData D;
  std::string err;
  // coarse level: single vertex patch (n_coarse == 2) or dense solve
  bool dense_coarse = false;
  int n_int_coarse = 0;
  std::vector<double> coarse_inv_host;  // n_int^2, FP64
  std::vector<int> coarse_coord;        // (x, y, z) of each interior coarse DoF
  VcycleVectors vc[2];  // [0] FP64, [1] FP32
  std::vector<int> sm_variant[2];  // per level: 3D smoother patches-per-batch variant (autotuned)
  std::vector<int> op_layers[2];   // per level: 3D operator cell layers per CTA (autotuned; 0 default)
  DevBuf dot_part;                 // 3D: per-CTA p.q partial sums of the fused CG operator
  int dot_cap = 0;                 // their capacity
  DevBuf err_flag;      // set by a kernel whose bounded wait gave up
  Mailbox mbox;         // small device results (CG scalars, dots, the error flag) for the host
  // variable coefficient: per-level per-cell kappa (fine given, coarse = mean of children)
  bool has_kappa = false;
  std::vector<std::vector<double>> kappa_host;
  std::vector<std::unique_ptr<DevBuf>> kappa_dev[2];  // [FP64, FP32][level]
  // Krylov work vectors (fine level, FP64)
  DevBuf r, p, q, partial, scalars;
  std::vector<std::unique_ptr<DevBuf>> gmres_v;
  // CUDA graph of one CG iteration
  cudaGraphExec_t graph = nullptr;
  int graph_key = -1;
  int tc_passes = 1;  // tensor-core smoother: 1 TF32 pass, 3 the three-term TF32 split
  cudaStream_t graph_stream = nullptr;
  const double *graph_x = nullptr;  // the captured graph updates this solution vector
  cudaStream_t own_stream = nullptr;  // used by tps_solve_host
  DevBuf host_b, host_x;              // device staging of tps_solve_host (kept, so its graph stays valid)
  // tps_solve_host_many: copy stream, double-buffered inputs and outputs, events
  cudaStream_t copy_stream = nullptr;
  DevBuf pipe_b[2], pipe_x[2];
  cudaEvent_t pipe_in[2] = {nullptr, nullptr}, pipe_done[2] = {nullptr, nullptr}, pipe_out[2] = {nullptr, nullptr};
  std::vector<std::unique_ptr<DevBuf>> fmg_sol, fmg_res;  // FMG: FP64 per level (lexicographic)
  DevBuf fmg_tmp;                                        // FMG: FP64 transfer scratch
  DevBuf adj_g, adj_lam;                                 // tps_adjoint: its right-hand side and lambda
  DevBuf var_r[2];      // separate-kernel smoother variants: residual of the finest-level size
  DevBuf var_acc[2];    // additive step: the summed patch solves
  int sm_kind = TPS_SMOOTHER_FUSED;  // V-cycle smoothing on levels >= 1
  double add_omega = 0.0;            // additive damping (0: 1/2^dim)
  DevBuf dense_inv[2];  // Exact variant: reference-cell interior patch inverse [FP64, FP32]
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;

  ~tps_handle()
  {
    if (graph) cudaGraphExecDestroy(graph);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (own_stream) cudaStreamDestroy(own_stream);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    for (int i = 0; i < 2; ++i) {
      if (pipe_in[i]) cudaEventDestroy(pipe_in[i]);
      if (pipe_done[i]) cudaEventDestroy(pipe_done[i]);
      if (pipe_out[i]) cudaEventDestroy(pipe_out[i]);
    }
  }
  const LevelGeomH &fine() const { return lv.back(); }
};

namespace {

int dt_index(int dtype)
{
  if (dtype != TPS_F64 && dtype != TPS_F32) throw ApiError(TPS_ERR_INVALID, "dtype must be TPS_F64 or TPS_F32");
  return dtype;
}

void check_level(const tps_handle *h, int level, int min_level = 0)
{
  if (level < min_level || level >= h->n_levels)
    throw ApiError(TPS_ERR_INVALID, "level " + std::to_string(level) + " out of range");
}

template <typename F>
int guarded(tps_handle *h, F &&f)
{
  if (!h) {
    g_create_error = "null handle";
    return TPS_ERR_INVALID;
  }
  try {
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) throw ApiError(TPS_ERR_CUDA, cudaGetErrorString(e));
    f();
    h->err.clear();
    return TPS_OK;
  } catch (const ApiError &e) {
    h->err = e.what();
    return e.code;
  } catch (const std::bad_alloc &) {
    h->err = "host allocation failed";
    return TPS_ERR_ALLOC;
  } catch (const std::exception &e) {
    h->err = e.what();
    return TPS_ERR_INVALID;
  }
}

// dense interior operator of the coarse level, assembled cell by cell on the
// host in FP64 (with the coarse-level kappa when present), and its inverse
void build_dense_coarse(tps_handle *h)
{
  const int k = h->k, n = h->n_coarse, N1 = n * k + 1, dim = h->dim;
  const double hh = 1.0 / n, s = stiffness_scale(dim, hh);
  const int np = k + 1;
  std::vector<int> idx1;
  for (int i = 1; i < N1 - 1; ++i) idx1.push_back(i);
  const int m1 = static_cast<int>(idx1.size());
  const int ni = dim == 3 ? m1 * m1 * m1 : m1 * m1;
  h->n_int_coarse = ni;
  auto coord = [&](int i, int &x, int &y, int &z) {
    x = idx1[i % m1];
    y = idx1[(i / m1) % m1];
    z = dim == 3 ? idx1[i / (m1 * m1)] : 0;
  };
  // interior index of a global coarse DoF (-1 on the boundary)
  auto interior = [&](int x, int y, int z) -> int {
    if (x < 1 || x > N1 - 2 || y < 1 || y > N1 - 2) return -1;
    if (dim == 3 && (z < 1 || z > N1 - 2)) return -1;
    return (x - 1) + (y - 1) * m1 + (dim == 3 ? (z - 1) * m1 * m1 : 0);
  };
  std::vector<double> A(static_cast<size_t>(ni) * ni, 0.0);
  const int ncell = dim == 3 ? n * n * n : n * n;
  const int csz = dim == 3 ? np * np * np : np * np;
  for (int c = 0; c < ncell; ++c) {
    const int cx = c % n, cy = (c / n) % n, cz = dim == 3 ? c / (n * n) : 0;
    const double kc = h->has_kappa ? h->kappa_host[0][c] : 1.0;
    for (int a = 0; a < csz; ++a) {
      const int ax = a % np, ay = (a / np) % np, az = dim == 3 ? a / (np * np) : 0;
      const int ia = interior(cx * k + ax, cy * k + ay, cz * k + az);
      if (ia < 0) continue;
      for (int b2 = 0; b2 < csz; ++b2) {
        const int bx = b2 % np, by = (b2 / np) % np, bz = dim == 3 ? b2 / (np * np) : 0;
        const int ib = interior(cx * k + bx, cy * k + by, cz * k + bz);
        if (ib < 0) continue;
        const double mx = h->D.cmass[ax * np + bx], my = h->D.cmass[ay * np + by];
        const double lx = h->D.clap[ax * np + bx], ly = h->D.clap[ay * np + by];
        double v;
        if (dim == 2) {
          v = ly * mx + my * lx;
        } else {
          const double mz = h->D.cmass[az * np + bz], lz = h->D.clap[az * np + bz];
          v = lz * my * mx + mz * ly * mx + mz * my * lx;
        }
        A[static_cast<size_t>(ia) * ni + ib] += kc * s * v;
      }
    }
  }
  // explicit inverse (coarse systems hold at most a few thousand DoFs)
  std::vector<double> inv;
  try {
    inv = spd_inverse(A, ni);
  } catch (const std::runtime_error &) {
    throw ApiError(TPS_ERR_INVALID, "coarse operator not positive definite");
  }
  h->coarse_inv_host = std::move(inv);
  h->coarse_coord.resize(3 * static_cast<size_t>(ni));
  for (int i = 0; i < ni; ++i) coord(i, h->coarse_coord[3 * i], h->coarse_coord[3 * i + 1],
                                     h->coarse_coord[3 * i + 2]);
}

VecLayout lex_layout(const tps_handle *h, int level)
{
  const int N1 = h->lv[level].N1;
  return VecLayout{N1, N1, int64_t(N1) * N1};
}

VcycleVectors &vcycle_vectors(tps_handle *h, int p)
{
  VcycleVectors &V = h->vc[p];
  if (V.ready) return V;
  const size_t es = p == 0 ? sizeof(double) : sizeof(float);
  const int align = static_cast<int>(16 / es);
  V.d.clear();
  V.su.clear();
  V.t.clear();
  V.tmp.clear();
  V.layout.clear();
  V.maps.assign(h->n_levels, SmootherMaps{});
  if (!h->err_flag.p) h->err_flag.alloc(sizeof(int));
  for (int l = 0; l < h->n_levels; ++l) {
    const LevelGeomH &g = h->lv[l];
    VecLayout lay;
    lay.N1 = g.N1;
    lay.sy = h->dim == 3 ? (g.N1 + align - 1) / align * align : g.N1;
    lay.sz = lay.sy * g.N1;
    const size_t n = static_cast<size_t>(h->dim == 3 ? lay.sz * g.N1 : lay.sy * g.N1);
    V.layout.push_back(lay);
    V.d.emplace_back(new DevBuf);
    V.su.emplace_back(new DevBuf);
    V.t.emplace_back(new DevBuf);
    V.tmp.emplace_back(new DevBuf);
    V.d[l]->alloc(es * n);
    V.su[l]->alloc(es * n);
    V.t[l]->alloc(es * n);
    if (l > 0 && h->dim == 3) {
      // transfer scratch: fine z x coarse y x coarse x
      const int64_t N1c = h->lv[l - 1].N1;
      V.tmp[l]->alloc(es * static_cast<size_t>(g.N1) * N1c * N1c);
    }
    if (h->dim == 3)
      TPS_CUDA(h->kt->encode_maps[p](lay, V.su[l]->p, V.d[l]->p, &V.maps[l]));
    if (h->dim == 3 && p == 1)
      TPS_CUDA(h->kt->encode_tc_maps(lay, V.su[l]->p, V.d[l]->p, &V.maps[l]));
  }
  if (h->dense_coarse) {
    const VecLayout &lc = V.layout[0];
    const int ni = h->n_int_coarse;
    std::vector<int> gidx(ni);
    for (int i = 0; i < ni; ++i)
      gidx[i] = static_cast<int>(h->coarse_coord[3 * i] + h->coarse_coord[3 * i + 1] * lc.sy +
                                 h->coarse_coord[3 * i + 2] * lc.sz);
    V.coarse_idx.alloc(sizeof(int) * ni);
    TPS_CUDA(cudaMemcpy(V.coarse_idx.p, gidx.data(), sizeof(int) * ni, cudaMemcpyHostToDevice));
  }
  if (h->dense_coarse) {
    const size_t n2 = h->coarse_inv_host.size();
    V.coarse_inv.alloc(es * n2);
    if (p == 0) {
      TPS_CUDA(cudaMemcpy(V.coarse_inv.p, h->coarse_inv_host.data(), es * n2, cudaMemcpyHostToDevice));
    } else {
      std::vector<float> f(n2);
      for (size_t i = 0; i < n2; ++i) f[i] = static_cast<float>(h->coarse_inv_host[i]);
      TPS_CUDA(cudaMemcpy(V.coarse_inv.p, f.data(), es * n2, cudaMemcpyHostToDevice));
    }
  }
  V.ready = true;
  return V;
}

// smoother variant of a level that was neither autotuned nor set.  FP32,
// degrees 2..4: two patches per warp in packed FP32 (variant 4) when a
// colour holds at least 4096 patches, else one warp per patch (variant 3).
// FP64 (and FP32 at other degrees): one warp per patch for degrees 3 and 4
// from 4096 patches per colour, else the default CTA batch.  Measured on B200
// (us per FP32 sweep, CTA batch / one warp per patch / two patches per warp):
// Q4 64^3 724 / 566 / 506, Q4 32^3 118 / 97 / 94, Q3 64^3 344 / 316 / 269,
// Q3 32^3 72 / 65 / 62, Q2 64^3 145 / 156 / 108, Q2 16^3 34 / 22 / 23;
// degree 5 is fastest with the CTA batch (248 / 310 / 307 at 32^3: the larger
// per-warp stages leave few warps per SM).  FP64: Q4 64^3 1166 vs 1052 (CTA
// batch vs one warp per patch), Q3 32^3 114 vs 105; 16^3 and coarser levels
// are launch-latency-bound and equal or faster with CTA batches.
int default_variant(const tps_handle *h, int level, int p)
{
  if (h->dim != 3) return 0;
  const int64_t c = h->lv[level].n / 2;  // patches per direction of colour 0
  const int64_t c3 = c * c * c;
  const bool large = c3 >= 4096, medium = c3 >= 512;
  const bool warp = h->kt->smoother_ppb(3, p == 0 ? 0 : 1, 3) == -1;  // one warp per patch compiled
  const bool pair = p == 1 && h->kt->smoother_ppb(3, 1, 4) == -2;     // two patches per warp compiled
  // The fastest variant per level size, measured on B200 (us per sweep,
  // variants 0..4 = CTA batch P, P/2, P/4, warp per patch, pair of patches):
  //   FP32 Q4 32^3 118 / 116 / 116 / 92 / 87, 16^3 37.2 / 37.5 / 39.4 / 38.9 / 35.4,
  //        8^3 36.3 / 31.4 / 33.8 / 36.4 / 31.4, 4^3 35.9 / 32.0 / 33.9 / 36.8 / 32.4;
  //   FP32 Q3 32^3 72 / 63 / 65 / 57 / 58, 16^3 34.6 / 27.1 / 27.5 / 29.8 / 32.0;
  //   FP32 Q2 16^3 34.4 / 27.9 / 25.2 / 21.9 / 23.0;
  //   FP64 Q4 32^3 165 / 171 / 165 / 135, 16^3 45.8 / 49.4 / 45.8 / 40.7,
  //        8^3 38.3 / 42.6 / 38.4 / 33.6, 4^3 38.8 / 42.7 / 38.8 / 33.1;
  //   FP64 Q3 32^3 98 / 96 / 101 / 80, 16^3 33.3 / 32.2 / 32.1 / 35.2, 8^3 32.2 / 28.8 / 27.4 / 31.5;
  //   FP64 Q2 32^3 41.4 / 41.2 / 40.8 / 42.6, 16^3 31.4 / 27.9 / 24.3 / 24.7.
  // Levels whose colours hold few patches are latency-bound; there the
  // smaller CTA batches win.
  if (p == 1) {
    if (pair && h->k >= 2 && h->k <= 4 && (large || (medium && h->k == 4))) return 4;
    if (warp && h->k == 2 && medium) return 3;
    return large ? 0 : 1;
  }
  if (warp && (h->k == 4 || (h->k == 3 && large))) return 3;
  if (h->k == 2 || h->k == 3) return 2;
  return 0;
}

// one coloured sweep; x_zero declares x == 0 on entry (the first colour then
// skips reading x); maps (may be null) select the TMA path; tc selects the
// tensor-core kernel (3D, FP32 vectors, constant coefficient, TMA views)
void smoother_sweep(tps_handle *h, int level, int p, const VecLayout &lay, void *x, const void *b,
                    bool reverse, bool x_zero, const SmootherMaps *maps, cudaStream_t s,
                    bool tc = false)
{
  const bool use_tc = tc && p == 1 && h->dim == 3 && !h->has_kappa && maps && maps->tc_valid &&
                      h->kt->smoother_tc;
  const int variant = level < static_cast<int>(h->sm_variant[p].size()) ? h->sm_variant[p][level]
                                                                        : default_variant(h, level, p);
  if (!h->err_flag.p) h->err_flag.alloc(sizeof(int));
  const int nc = 1 << h->dim;
  for (int i = 0; i < nc; ++i) {
    const int c = reverse ? nc - 1 - i : i;
    if (h->has_kappa)
      TPS_CUDA(h->kt->kappa_smoother[h->dim - 2][p](h->lv[level], lay, x, b,
                                                    h->kappa_dev[p][level]->p, c, h->omega, s));
    else if (use_tc)
      TPS_CUDA(h->kt->smoother_tc(h->lv[level], lay, x, b, c, h->omega, (x_zero && i == 0) ? 1 : 0, maps,
                                  h->tc_passes, h->err_flag.as<int>(), s));
    else
      TPS_CUDA(h->kt->smoother[h->dim - 2][p](h->lv[level], lay, x, b, c, h->omega,
                                              (x_zero && i == 0) ? 1 : 0, variant, maps,
                                              h->err_flag.as<int>(), s));
  }
}

// level operator: dst = A src (mode 0, interior rows) or rhs - A src (mode 1)
void level_laplace(tps_handle *h, int level, int p, const VecLayout &lay, void *dst, const void *src,
                   const void *rhs, int mode, cudaStream_t s)
{
  if (h->has_kappa)
    TPS_CUDA(h->kt->kappa_laplace[h->dim - 2][p](h->lv[level], lay, dst, src, rhs,
                                                 h->kappa_dev[p][level]->p, mode, s));
  else
    TPS_CUDA(h->kt->laplace[h->dim - 2][p](h->lv[level], lay, dst, src, rhs, mode,
                                           level < static_cast<int>(h->op_layers[p].size())
                                               ? h->op_layers[p][level] : 0,
                                           s));
}

// per-level coefficients from the finest-level kappa (coarse = mean of the 2^d
// children).  Built aside and committed at the end: a rejected kappa or a failed
// allocation leaves the handle's coefficients as they were.
void set_kappa_levels(tps_handle *h, const double *kappa_fine)
{
  const int L = h->n_levels - 1, dim = h->dim;
  const int64_t ncf = dim == 3 ? int64_t(h->lv[L].n) * h->lv[L].n * h->lv[L].n
                               : int64_t(h->lv[L].n) * h->lv[L].n;
  for (int64_t c = 0; c < ncf; ++c)
    if (!(kappa_fine[c] > 0.0) || !std::isfinite(kappa_fine[c]))
      throw ApiError(TPS_ERR_INVALID, "kappa must be positive and finite");
  std::vector<std::vector<double>> kh(h->n_levels);
  kh[L].assign(kappa_fine, kappa_fine + ncf);
  for (int l = L - 1; l >= 0; --l) {
    const int n = h->lv[l].n, nf = h->lv[l + 1].n;
    const int64_t nc = dim == 3 ? int64_t(n) * n * n : int64_t(n) * n;
    kh[l].assign(nc, 0.0);
    for (int64_t c = 0; c < nc; ++c) {
      const int cx = int(c % n), cy = int((c / n) % n), cz = dim == 3 ? int(c / (int64_t(n) * n)) : 0;
      double acc = 0.0;
      for (int q = 0; q < (1 << dim); ++q) {
        const int fx = 2 * cx + (q & 1), fy = 2 * cy + ((q >> 1) & 1), fz = 2 * cz + ((q >> 2) & 1);
        acc += kh[l + 1][fx + int64_t(fy) * nf + (dim == 3 ? int64_t(fz) * nf * nf : 0)];
      }
      kh[l][c] = acc / (1 << dim);
    }
  }
  // the device buffers are allocated once and then rewritten in place, so
  // captured graphs (the CG iteration, a batch) keep valid pointers
  if (h->kappa_dev[1].size() != static_cast<size_t>(h->n_levels)) {
    std::vector<std::unique_ptr<DevBuf>> kd[2];
    for (int p = 0; p < 2; ++p)
      for (int l = 0; l < h->n_levels; ++l) {
        kd[p].emplace_back(new DevBuf);
        kd[p][l]->alloc((p == 0 ? sizeof(double) : sizeof(float)) * kh[l].size());
      }
    for (int p = 0; p < 2; ++p) h->kappa_dev[p] = std::move(kd[p]);
  }
  for (int l = 0; l < h->n_levels; ++l) {
    const size_t nc = kh[l].size();
    TPS_CUDA(cudaMemcpy(h->kappa_dev[0][l]->p, kh[l].data(), sizeof(double) * nc, cudaMemcpyHostToDevice));
    const std::vector<float> f(kh[l].begin(), kh[l].end());
    TPS_CUDA(cudaMemcpy(h->kappa_dev[1][l]->p, f.data(), sizeof(float) * nc, cudaMemcpyHostToDevice));
  }
  h->kappa_host = std::move(kh);
}

void coarse_solve(tps_handle *h, int p, cudaStream_t s, bool tc)
{
  VcycleVectors &V = h->vc[p];
  const size_t es = p == 0 ? sizeof(double) : sizeof(float);
  const VecLayout &lay = V.layout[0];
  TPS_CUDA(cudaMemsetAsync(V.su[0]->p, 0, es * V.su[0]->bytes / es, s));
  if (!h->dense_coarse) {
    // one vertex patch covers every interior DoF: the smoother is an exact solve
    smoother_sweep(h, 0, p, lay, V.su[0]->p, V.d[0]->p, false, true, &V.maps[0], s, tc);
  } else {
    TPS_CUDA(launch_coarse_dense(V.coarse_inv.p, V.coarse_idx.as<int>(), h->n_int_coarse,
                                 V.su[0]->p, V.d[0]->p, static_cast<int>(es), s));
  }
}

// entries of a level vector in layout lay, row padding included
int64_t layout_elems(const tps_handle *h, const VecLayout &lay)
{
  return h->dim == 3 ? lay.sz * lay.N1 : lay.sy * lay.N1;
}

// the additive step's scratch vectors of precision p, sized for the finest
// level in any layout (rows are padded by fewer than 4 entries); allocated
// before any graph capture by tps_set_smoother_kind
void ensure_additive_scratch(tps_handle *h, int p)
{
  const int64_t N1 = h->fine().N1;
  const int64_t n = h->dim == 3 ? (N1 + 4) * N1 * N1 : (N1 + 4) * N1;
  const size_t bytes = (p == 0 ? 8 : 4) * static_cast<size_t>(n);
  if (h->var_r[p].bytes < bytes) h->var_r[p].alloc(bytes);
  if (h->var_acc[p].bytes < bytes) h->var_acc[p].alloc(bytes);
}

double additive_omega(const tps_handle *h) { return h->add_omega > 0 ? h->add_omega : 1.0 / (1 << h->dim); }

// Additive vertex-patch Schwarz step (no reference counterpart; the
// reference's sweep is the coloured multiplicative one): r = b - A x (r = b
// when x == 0), acc = the sum over all patches of A_II^{-1} r_I (the patch
// solve with omega 1 adds into the zeroed acc colour by colour, so no two
// writes of one launch meet: deterministic), x += omega acc.
void additive_sweep(tps_handle *h, int level, int p, const VecLayout &lay, void *x, const void *b, bool x_zero,
                    cudaStream_t s)
{
  if (h->has_kappa) throw ApiError(TPS_ERR_UNSUPPORTED, "the additive step has a constant coefficient");
  ensure_additive_scratch(h, p);
  const LevelGeomH &g = h->lv[level];
  const size_t es = p == 0 ? 8 : 4;
  const int64_t n = layout_elems(h, lay);
  const void *r = b;
  if (!x_zero) {
    level_laplace(h, level, p, lay, h->var_r[p].p, x, b, 1, s);
    r = h->var_r[p].p;
  }
  TPS_CUDA(cudaMemsetAsync(h->var_acc[p].p, 0, es * static_cast<size_t>(n), s));
  for (int c = 0; c < (1 << h->dim); ++c)
    TPS_CUDA(h->kt->patch_solve[h->dim - 2][p](g, lay, h->var_acc[p].p, r, nullptr, c, 1.0, s));
  TPS_CUDA(h->kt->scaled_add[p](x, h->var_acc[p].p, additive_omega(h), n, s));
}

// the V-cycle's smoothing on levels >= 1: the additive step when selected
void level_smooth(tps_handle *h, int level, int p, const VecLayout &lay, void *x, const void *b, bool reverse,
                  bool x_zero, const SmootherMaps *maps, cudaStream_t s, bool tc)
{
  if (h->sm_kind == TPS_SMOOTHER_ADDITIVE)
    additive_sweep(h, level, p, lay, x, b, x_zero, s);
  else
    smoother_sweep(h, level, p, lay, x, b, reverse, x_zero, maps, s, tc);
}

// MultigridSolvers::v_cycle (include/solver.cuh:1952-2001) on precision p:
// input d[level], output su[level]; tc: FP32 3D sweeps on the tensor cores;
// zero_init = false continues from the current su[level] (a further cycle of
// v_cycle(level, n_cycles), include/solver.cuh:798-805)
// Inside the TF32 V-cycle the tensor-core smoother runs a level only where it
// is faster than the FP32 SIMT kernels: degrees 2..4 (the patch-GEMM kernel)
// on levels whose colour 0 fills a wave of 128-patch tiles on every SM.
// Smaller levels are latency-bound and keep the SIMT smoother.
bool tc_pays(const tps_handle *h, int level)
{
  if (h->dim != 3 || h->k > 4 || (h->tc_passes == 3 && h->k != 4)) return false;
  const int64_t c = h->lv[level].n / 2;
  return c * c * c >= 128 * static_cast<int64_t>(h->n_sm);
}

void vcycle_rec(tps_handle *h, int level, int p, bool symmetric, cudaStream_t s, bool tc,
                bool zero_init = true)
{
  static const char *const kLevelNames[] = {"V-cycle level 0", "V-cycle level 1", "V-cycle level 2",
                                            "V-cycle level 3", "V-cycle level 4", "V-cycle level 5",
                                            "V-cycle level 6", "V-cycle level 7", "V-cycle level 8",
                                            "V-cycle level 9", "V-cycle level 10", "V-cycle level 11"};
  TPS_RANGE(kLevelNames[level < 12 ? level : 11]);
  VcycleVectors &V = h->vc[p];
  if (level == 0) {
    coarse_solve(h, p, s, tc && tc_pays(h, 0));
    return;
  }
  const LevelGeomH &g = h->lv[level];
  const VecLayout &lay = V.layout[level], &lc = V.layout[level - 1];
  const int di = h->dim - 2;
  if (zero_init) TPS_CUDA(cudaMemsetAsync(V.su[level]->p, 0, V.su[level]->bytes, s));
  const bool tcl = tc && tc_pays(h, level);
  level_smooth(h, level, p, lay, V.su[level]->p, V.d[level]->p, false, zero_init, &V.maps[level], s, tcl);
  level_laplace(h, level, p, lay, V.t[level]->p, V.su[level]->p, V.d[level]->p, 1, s);
  TPS_CUDA(h->kt->restrict_[di][p](h->lv[level - 1], lc, lay, V.d[level - 1]->p, V.t[level]->p,
                                   V.tmp[level]->p, 0, s));
  vcycle_rec(h, level - 1, p, symmetric, s, tc);
  TPS_CUDA(h->kt->prolong[di][p](h->lv[level - 1], lc, lay, V.su[level]->p, V.su[level - 1]->p,
                                 V.tmp[level]->p, s));
  level_smooth(h, level, p, lay, V.su[level]->p, V.d[level]->p, symmetric, false, &V.maps[level], s, tcl);
}

int vprec_index(int precision)
{
  if (precision < 0 || precision > 4) throw ApiError(TPS_ERR_INVALID, "bad V-cycle precision");
  return precision == TPS_VCYCLE_F32 || precision == TPS_VCYCLE_TF32 || precision == TPS_VCYCLE_TF32X3 ? 1 : 0;
}
// conversion of the FP64 input into the V-cycle vectors: 0 f64, 1 f32, 2 f64-rounded
int input_kind(int precision)
{
  return precision == TPS_VCYCLE_TF32 || precision == TPS_VCYCLE_TF32X3 ? 1 : precision;
}
bool vprec_tc(int precision) { return precision == TPS_VCYCLE_TF32 || precision == TPS_VCYCLE_TF32X3; }
// tensor-core passes of a V-cycle precision (only read where vprec_tc holds)
int vprec_passes(int precision) { return precision == TPS_VCYCLE_TF32X3 ? 3 : 1; }

// the tensor-core smoother exists for 3D, degree >= 2, constant coefficient;
// records the passes (1 TF32, 3 the three-term split) for the sweeps that follow
void check_tc(tps_handle *h, int passes = 1)
{
  if (h->dim != 3 || !h->kt->smoother_tc || h->has_kappa)
    throw ApiError(TPS_ERR_UNSUPPORTED, "the tensor-core (TF32) smoother needs 3D, degree >= 2 and no kappa");
  h->tc_passes = passes;
}


PadMap fine_padmap(tps_handle *h, int p)
{
  const VecLayout &l = h->vc[p].layout.back();
  return make_padmap(l.N1, l.sy);
}

void fine_vmult64(tps_handle *h, double *dst, const double *src, cudaStream_t s)
{
  const LevelGeomH &g = h->fine();
  level_laplace(h, h->n_levels - 1, 0, lex_layout(h, h->n_levels - 1), dst, src, nullptr, 0, s);
  TPS_CUDA(launch_copy_boundary(dst, src, h->dim, g.N1, 8, s));
}

// `bytes` (a multiple of 4, at most 256) of device memory at src, read on
// stream s after the work queued there: a one-warp kernel stores them into the
// handle's host-mapped mailbox, then the stream is synchronized
void read_small(tps_handle *h, void *out, const void *src, size_t bytes, cudaStream_t s)
{
  h->mbox.ensure();
  void *dst = nullptr;
  TPS_CUDA(cudaHostGetDevicePointer(&dst, h->mbox.host, 0));
  TPS_CUDA(launch_copy_words(src, dst, static_cast<int>(bytes / 4), s));
  TPS_CUDA(cudaStreamSynchronize(s));
  std::memcpy(out, h->mbox.host, bytes);
}

// Reads and clears the handle's device error flag once the work queued on `s`
// is done; true when a bounded device wait of an earlier launch ran out.
bool take_timeout_flag(tps_handle *h, cudaStream_t s)
{
  if (!h->err_flag.p) return false;
  int v = 0;
  read_small(h, &v, h->err_flag.p, sizeof(int), s);
  if (v == 0) return false;
  TPS_CUDA(cudaMemsetAsync(h->err_flag.p, 0, sizeof(int), s));
  TPS_CUDA(cudaStreamSynchronize(s));
  return true;
}

// message of a status that a call returns without throwing ("" for TPS_OK)
const char *status_message(int status)
{
  switch (status) {
    case TPS_ERR_NOT_CONVERGED: return "solver did not converge within max_iter";
    case TPS_ERR_BREAKDOWN: return "Krylov breakdown (p^T A p <= 0)";
    case TPS_ERR_NONFINITE: return "non-finite residual";
    case TPS_ERR_TIMEOUT:
      return "a bounded device wait ran out (a staged copy did not complete); results since the last check are invalid";
    default: return "";
  }
}

void ensure_krylov(tps_handle *h)
{
  const int64_t N = h->fine().N;
  // each buffer on its own: one whose allocation failed is retried next time
  if (!h->r.p) h->r.alloc(sizeof(double) * N);
  if (!h->p.p) h->p.alloc(sizeof(double) * N);
  if (!h->q.p) h->q.alloc(sizeof(double) * N);
  if (!h->partial.p) h->partial.alloc(sizeof(double) * kRedBlocks * 4);
  if (!h->scalars.p) h->scalars.alloc(sizeof(CGScalars) + 64);
  if (h->dim == 3 && !h->dot_part.p) {
    h->dot_cap = h->kt->laplace3d_ctas(h->fine().n);
    h->dot_part.alloc(sizeof(double) * h->dot_cap);
  }
  if (!h->ev0) {
    TPS_CUDA(cudaEventCreate(&h->ev0));
    TPS_CUDA(cudaEventCreate(&h->ev1));
  }
}

// q = A p on the finest level and alpha = rz / p.q; in 3D without a
// coefficient the operator kernel forms the p.q partial sums itself
void cg_q_alpha(tps_handle *h, const VecLayout &lex, cudaStream_t s)
{
  const int L = h->n_levels - 1;
  CGScalars *sc = h->scalars.as<CGScalars>();
  if (h->dim == 3 && !h->has_kappa && h->dot_part.p) {
    int ctas = 0;
    const int layers = L < static_cast<int>(h->op_layers[0].size()) ? h->op_layers[0][L] : 0;
    TPS_CUDA(h->kt->laplace3d_dot(h->lv[L], lex, h->q.p, h->p.p, h->dot_part.as<double>(), h->dot_cap, layers,
                                  &ctas, s));
    TPS_CUDA(launch_cg_alpha_partials(h->dot_part.as<double>(), ctas, sc, s));
  } else {
    level_laplace(h, L, 0, lex, h->q.p, h->p.p, nullptr, 0, s);
    TPS_CUDA(launch_cg_alpha(h->p.as<double>(), h->q.as<double>(), h->fine().N, h->partial.as<double>(), sc, s));
  }
}

// the part of a CG iteration that follows the convergence check:
// z = V(d); beta; p = z + beta p; q = A p; alpha; x, r update; rr
void cg_iteration_body(tps_handle *h, int prec, bool symmetric, double *x, cudaStream_t s)
{
  const int p = vprec_index(prec);
  const int L = h->n_levels - 1;
  const int64_t N = h->fine().N;
  VcycleVectors &V = h->vc[p];
  CGScalars *sc = h->scalars.as<CGScalars>();
  double *part = h->partial.as<double>();
  const int zk = p == 1 ? 1 : 0;
  const PadMap pm = fine_padmap(h, p);
  const VecLayout lex = lex_layout(h, L);
  vcycle_rec(h, L, p, symmetric, s, vprec_tc(prec));
  TPS_CUDA(launch_cg_beta(V.su[L]->p, zk, pm, h->q.as<double>(), h->r.as<double>(), N, part, sc, s));
  TPS_CUDA(launch_cg_update_p(h->p.as<double>(), V.su[L]->p, zk, pm, N, sc, s));
  cg_q_alpha(h, lex, s);
  TPS_CUDA(launch_cg_update_xr(x, h->r.as<double>(), h->p.as<double>(), h->q.as<double>(),
                               V.d[L]->p, input_kind(prec), pm, N, part, sc, s));
  TPS_CUDA(launch_cg_finalize_rr(part, sc, s));
}

static_assert(sizeof(CGScalars) % 4 == 0 && sizeof(CGScalars) <= Mailbox::kBytes, "CG scalars fit the mailbox");

void read_scalars(tps_handle *h, CGScalars &out, cudaStream_t s)
{
  read_small(h, &out, h->scalars.p, sizeof(CGScalars), s);
}

int solve_cg(tps_handle *h, const tps_solve_opts &o, const double *b, double *x, tps_report *rep,
             cudaStream_t s)
{
  TPS_RANGE("tps_solve CG");
  const int p = vprec_index(o.precision);
  if (vprec_tc(o.precision)) check_tc(h, vprec_passes(o.precision));
  vcycle_vectors(h, p);
  ensure_krylov(h);
  const int L = h->n_levels - 1;
  const LevelGeomH &g = h->fine();
  const int64_t N = g.N;
  VcycleVectors &V = h->vc[p];
  CGScalars *sc = h->scalars.as<CGScalars>();
  double *part = h->partial.as<double>();
  const int zk = p == 1 ? 1 : 0;
  const bool sym = o.symmetric != 0;
  const PadMap pm = fine_padmap(h, p);
  const VecLayout lex = lex_layout(h, L);
  TPS_CUDA(cudaEventRecord(h->ev0, s));
  // Dirichlet rows: x_b = b_b, so r_b = 0 and the iteration lives on the interior
  TPS_CUDA(launch_copy_boundary(x, b, h->dim, g.N1, 8, s));
  TPS_CUDA(cudaMemsetAsync(h->r.p, 0, sizeof(double) * N, s));
  TPS_CUDA(cudaMemsetAsync(h->q.p, 0, sizeof(double) * N, s));
  level_laplace(h, L, 0, lex, h->r.p, x, b, 1, s);
  TPS_CUDA(launch_cg_init(h->r.as<double>(), b, V.d[L]->p, input_kind(o.precision), pm, N, part, s));
  TPS_CUDA(launch_cg_finalize_init(part, sc, s));
  CGScalars hs{};
  read_scalars(h, hs, s);
  const double bnorm = std::sqrt(hs.bb) > 0 ? std::sqrt(hs.bb) : 1.0;
  double res = std::sqrt(hs.rr) / bnorm;
  rep->initial_residual = std::sqrt(hs.rr);
  rep->history[0] = res;
  int it = 0;
  int status = TPS_OK;
  if (hs.breakdown) status = TPS_ERR_NONFINITE;
  bool converged = res <= o.rel_tol;
  if (!converged && status == TPS_OK) {
    // first direction: z = V(r), p = z, rz; then q, alpha, x/r update
    vcycle_rec(h, L, p, sym, s, vprec_tc(o.precision));
    TPS_CUDA(launch_cg_first_direction(h->p.as<double>(), V.su[L]->p, zk, pm, h->r.as<double>(), N,
                                       part, s));
    TPS_CUDA(launch_cg_finalize_rz(part, sc, s));
    cg_q_alpha(h, lex, s);
    TPS_CUDA(launch_cg_update_xr(x, h->r.as<double>(), h->p.as<double>(), h->q.as<double>(),
                                 V.d[L]->p, input_kind(o.precision), pm, N, part, sc, s));
    TPS_CUDA(launch_cg_finalize_rr(part, sc, s));
    it = 1;
    const int key = (o.precision << 1) | (sym ? 1 : 0);
    // the graph bakes in x, so it is only reused for the same x pointer
    cudaGraphExec_t exec = nullptr;
    // stream capture is not available on the legacy default stream
    bool use_graph = o.use_graph != 0 && s != nullptr;
    for (;;) {
      TPS_RANGE("CG iteration");
      read_scalars(h, hs, s);
      res = std::sqrt(hs.rr) / bnorm;
      if (it < TPS_MAX_HISTORY) rep->history[it] = res;
      if (hs.breakdown) {
        status = hs.breakdown == 2 ? TPS_ERR_NONFINITE : TPS_ERR_BREAKDOWN;
        break;
      }
      if (res <= o.rel_tol) {
        converged = true;
        break;
      }
      if (it >= o.max_iter) break;
      if (use_graph) {
        if (!exec) {
          if (h->graph && h->graph_key == key && h->graph_stream == s && h->graph_x == x) {
            exec = h->graph;
          } else {
            if (h->graph) {
              cudaGraphExecDestroy(h->graph);
              h->graph = nullptr;
            }
            cudaGraph_t graph;
            TPS_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            try {
              cg_iteration_body(h, o.precision, sym, x, s);
            } catch (...) {
              cudaStreamEndCapture(s, &graph);
              throw;
            }
            TPS_CUDA(cudaStreamEndCapture(s, &graph));
            cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            TPS_CUDA(e);
            h->graph = exec;
            h->graph_key = key;
            h->graph_stream = s;
            h->graph_x = x;
          }
        }
        TPS_CUDA(cudaGraphLaunch(exec, s));
      } else {
        cg_iteration_body(h, o.precision, sym, x, s);
      }
      ++it;
    }
  }
  TPS_CUDA(cudaEventRecord(h->ev1, s));
  TPS_CUDA(cudaEventSynchronize(h->ev1));
  float ms = 0.f;
  TPS_CUDA(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  rep->time_ms = ms;
  rep->iterations = it;
  rep->final_residual = res;
  rep->converged = converged ? 1 : 0;
  if (status == TPS_OK && !converged) status = TPS_ERR_NOT_CONVERGED;
  return status;
}

double dev_dot(tps_handle *h, const double *a, const double *b, cudaStream_t s)
{
  double *part = h->partial.as<double>();
  TPS_CUDA(launch_dot_f64(a, b, h->fine().N, part, s));
  TPS_CUDA(launch_reduce(part, 1, part + 2 * kRedBlocks, s));
  double v = 0;
  read_small(h, &v, part + 2 * kRedBlocks, sizeof(double), s);
  return v;
}

// preconditioner application dst = V(src), FP64 in/out
void apply_vcycle64(tps_handle *h, int precision, bool symmetric, double *dst, const double *src,
                    cudaStream_t s)
{
  const int p = vprec_index(precision);
  if (vprec_tc(precision)) check_tc(h, vprec_passes(precision));
  VcycleVectors &V = vcycle_vectors(h, p);
  const int L = h->n_levels - 1;
  const int64_t N = h->fine().N;
  const PadMap pm = fine_padmap(h, p);
  TPS_CUDA(launch_to_vcycle(V.d[L]->p, input_kind(precision), pm, src, N, s));
  vcycle_rec(h, L, p, symmetric, s, vprec_tc(precision));
  TPS_CUDA(launch_from_vcycle(dst, V.su[L]->p, p == 1 ? 1 : 0, pm, N, s));
}


// best of three timed runs of fn on stream s (after one untimed run), ms
template <class F>
float best_of_three(tps_handle *h, cudaStream_t s, F &&fn)
{
  fn();
  float t = 1e30f;
  for (int r = 0; r < 3; ++r) {
    TPS_CUDA(cudaEventRecord(h->ev0, s));
    fn();
    TPS_CUDA(cudaEventRecord(h->ev1, s));
    TPS_CUDA(cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    TPS_CUDA(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    t = ms < t ? ms : t;
  }
  return t;
}

// Autotuner of the 3D level kernels of precision p, on the V-cycle work
// vectors: per level, the smoother's patches-per-batch variant (one sweep per
// candidate) and the operator's tile depth in z (cell layers per CTA of the
// z-marching kernel, one residual per candidate); the fastest of each is kept.
void autotune_levels(tps_handle *h, int p, cudaStream_t s)
{
  VcycleVectors &V = vcycle_vectors(h, p);
  ensure_krylov(h);
  h->sm_variant[p].assign(h->n_levels, 0);
  h->op_layers[p].assign(h->n_levels, 0);
  if (h->dim != 3 || h->has_kappa) return;
  for (int l = 0; l < h->n_levels; ++l) {
    float best_op = 1e30f;
    int bz = 0;
    for (int cz = 1; cz <= 16 && cz <= h->lv[l].n; cz *= 2) {
      h->op_layers[p][l] = cz;
      const float t = best_of_three(h, s, [&] {
        level_laplace(h, l, p, V.layout[l], V.t[l]->p, V.su[l]->p, V.d[l]->p, 1, s);
      });
      if (t < best_op) {
        best_op = t;
        bz = cz;
      }
    }
    h->op_layers[p][l] = bz;
  }
  for (int l = 0; l < h->n_levels; ++l) {
    float best = 1e30f;
    int bv = 0;
    for (int v = 0; v < kSmootherVariants; ++v) {
      if (v > 0 && h->kt->smoother_ppb(3, p == 0 ? 0 : 1, v) == h->kt->smoother_ppb(3, p == 0 ? 0 : 1, 0)) continue;
      h->sm_variant[p][l] = v;
      const float t = best_of_three(h, s, [&] {
        smoother_sweep(h, l, p, V.layout[l], V.su[l]->p, V.d[l]->p, false, false, &V.maps[l], s);
      });
      if (t < best) {
        best = t;
        bv = v;
      }
    }
    h->sm_variant[p][l] = bv;
  }
  TPS_CUDA(cudaMemsetAsync(V.su.back()->p, 0, V.su.back()->bytes, s));
}

// tps_smoother_step with TPS_TF32 on caller vectors (FP32, lexicographic):
// the sweep runs on the padded, TMA-addressable V-cycle vectors of the level
void tc_smoother_step(tps_handle *h, int level, void *x, const void *b, bool zero_init, bool reverse, int passes,
                      cudaStream_t s)
{
  check_tc(h, passes);
  if (passes == 3 && h->k != 4)
    throw ApiError(TPS_ERR_UNSUPPORTED, "the three-term TF32 tensor-core smoother needs degree 4");
  VcycleVectors &V = vcycle_vectors(h, 1);
  const VecLayout &l = V.layout[level];
  const size_t row = sizeof(float) * l.N1, pitch = sizeof(float) * l.sy;
  const size_t rows = static_cast<size_t>(l.N1) * l.N1;
  void *px = V.su[level]->p, *pb = V.d[level]->p;
  if (zero_init)
    TPS_CUDA(cudaMemsetAsync(px, 0, V.su[level]->bytes, s));
  else
    TPS_CUDA(cudaMemcpy2DAsync(px, pitch, x, row, row, rows, cudaMemcpyDeviceToDevice, s));
  TPS_CUDA(cudaMemcpy2DAsync(pb, pitch, b, row, row, rows, cudaMemcpyDeviceToDevice, s));
  smoother_sweep(h, level, 1, l, px, pb, reverse, zero_init, &V.maps[level], s, true);
  TPS_CUDA(cudaMemcpy2DAsync(x, row, px, pitch, row, rows, cudaMemcpyDeviceToDevice, s));
}

// MultigridSolvers::solve (include/solver.cuh:1784-1860), see tps_fmg
void fmg(tps_handle *h, int precision, int n_cycles, const double *const *rhs, const double *const *bnd,
         double *x, tps_report *rep, cudaStream_t s)
{
  TPS_RANGE("tps_fmg");
  const int p = vprec_index(precision), L = h->n_levels - 1, dim = h->dim;
  const bool tc = vprec_tc(precision);
  if (tc) check_tc(h, vprec_passes(precision));
  VcycleVectors &V = vcycle_vectors(h, p);
  ensure_krylov(h);
  if (h->fmg_sol.size() != static_cast<size_t>(h->n_levels)) {
    // built aside and kept only once every allocation succeeded
    std::vector<std::unique_ptr<DevBuf>> sol, res;
    size_t tmp = 0;
    for (int l = 0; l <= L; ++l) {
      sol.emplace_back(new DevBuf);
      res.emplace_back(new DevBuf);
      if (l < L) sol[l]->alloc(sizeof(double) * h->lv[l].N);
      res[l]->alloc(sizeof(double) * h->lv[l].N);
      if (l > 0 && dim == 3)
        tmp = std::max(tmp, sizeof(double) * static_cast<size_t>(h->lv[l].N1) * h->lv[l - 1].N1 * h->lv[l - 1].N1);
    }
    if (tmp) h->fmg_tmp.alloc(tmp);
    h->fmg_sol = std::move(sol);
    h->fmg_res = std::move(res);
  }
  auto padmap = [&](int l) { return make_padmap(V.layout[l].N1, V.layout[l].sy); };
  const int zk = p == 1 ? 1 : 0;
  TPS_CUDA(cudaEventRecord(h->ev0, s));
  // coarse level: coarse solve, then one more smoother step
  TPS_CUDA(launch_to_vcycle(V.d[0]->p, input_kind(precision), padmap(0), rhs[0], h->lv[0].N, s));
  coarse_solve(h, p, s, tc && tc_pays(h, 0));
  smoother_sweep(h, 0, p, V.layout[0], V.su[0]->p, V.d[0]->p, false, false, &V.maps[0], s, tc && tc_pays(h, 0));
  double *sol0 = L == 0 ? x : h->fmg_sol[0]->as<double>();
  TPS_CUDA(launch_from_vcycle(sol0, V.su[0]->p, zk, padmap(0), h->lv[0].N, s));
  for (int l = 1; l <= L; ++l) {
    const LevelGeomH &g = h->lv[l], &gc = h->lv[l - 1];
    double *solc = h->fmg_sol[l - 1]->as<double>();
    double *sol = l == L ? x : h->fmg_sol[l]->as<double>();
    double *res = h->fmg_res[l]->as<double>();
    if (bnd && bnd[l - 1]) TPS_CUDA(launch_copy_boundary(solc, bnd[l - 1], dim, gc.N1, 8, s));
    TPS_CUDA(cudaMemsetAsync(sol, 0, sizeof(double) * g.N, s));
    TPS_CUDA(h->kt->prolong_nb[dim - 2](gc, lex_layout(h, l - 1), lex_layout(h, l), sol, solc, h->fmg_tmp.p, s));
    TPS_CUDA(cudaMemsetAsync(res, 0, sizeof(double) * g.N, s));
    level_laplace(h, l, 0, lex_layout(h, l), res, sol, rhs[l], 1, s);
    TPS_CUDA(launch_to_vcycle(V.d[l]->p, input_kind(precision), padmap(l), res, g.N, s));
    for (int c = 0; c < n_cycles; ++c) vcycle_rec(h, l, p, false, s, tc, c == 0);
    TPS_CUDA(launch_from_vcycle(res, V.su[l]->p, zk, padmap(l), g.N, s));
    TPS_CUDA(launch_axpy_f64(sol, 1.0, res, g.N, s));
  }
  // final relative residual of the homogeneous part, then the Dirichlet data
  double *r = h->fmg_res[L]->as<double>();
  TPS_CUDA(cudaMemsetAsync(r, 0, sizeof(double) * h->fine().N, s));
  level_laplace(h, L, 0, lex_layout(h, L), r, x, rhs[L], 1, s);
  const double rr = dev_dot(h, r, r, s);
  // ||b|| on the interior rows: r = rhs - A 0 writes exactly those rows
  TPS_CUDA(cudaMemsetAsync(h->q.p, 0, sizeof(double) * h->fine().N, s));
  TPS_CUDA(cudaMemsetAsync(h->r.p, 0, sizeof(double) * h->fine().N, s));
  level_laplace(h, L, 0, lex_layout(h, L), h->r.p, h->q.p, rhs[L], 1, s);
  const double bb = dev_dot(h, h->r.as<double>(), h->r.as<double>(), s);
  if (bnd && bnd[L]) TPS_CUDA(launch_copy_boundary(x, bnd[L], dim, h->fine().N1, 8, s));
  TPS_CUDA(cudaEventRecord(h->ev1, s));
  TPS_CUDA(cudaEventSynchronize(h->ev1));
  float ms = 0.f;
  TPS_CUDA(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  if (rep) {
    std::memset(rep, 0, sizeof(*rep));
    rep->iterations = n_cycles;
    rep->initial_residual = std::sqrt(bb);
    rep->final_residual = std::sqrt(rr) / (bb > 0 ? std::sqrt(bb) : 1.0);
    rep->history[0] = 1.0;
    rep->converged = std::isfinite(rep->final_residual) ? 1 : 0;
    rep->time_ms = ms;
  }
}

// deal.II SolverGMRES semantics (left preconditioning, MGS, Givens) as used by
// MultigridSolvers::solve_gmres (include/solver.cuh:1865-1910)
int solve_gmres(tps_handle *h, const tps_solve_opts &o, const double *b, double *x,
                tps_report *rep, cudaStream_t s)
{
  TPS_RANGE("tps_solve GMRES");
  ensure_krylov(h);
  vcycle_vectors(h, vprec_index(o.precision));
  const LevelGeomH &g = h->fine();
  const int64_t N = g.N;
  const int basis = 28;  // max_n_tmp_vectors - 2 with deal.II's default of 30
  const int nvec = std::min(basis, std::max(o.max_iter, 1)) + 1;
  while (static_cast<int>(h->gmres_v.size()) < nvec) {
    std::unique_ptr<DevBuf> v(new DevBuf);
    v->alloc(sizeof(double) * N);
    h->gmres_v.push_back(std::move(v));
  }
  auto Vp = [&](int i) { return h->gmres_v[i]->as<double>(); };
  double *pv = h->p.as<double>();
  TPS_CUDA(cudaEventRecord(h->ev0, s));
  TPS_CUDA(launch_copy_boundary(x, b, h->dim, g.N1, 8, s));
  std::vector<double> H((basis + 1) * basis, 0.0), hv(basis + 1), gam(basis + 1), ci(basis + 1),
      si(basis + 1);
  int acc = 0, state = 0;  // 0 iterate, 1 success, 2 failure
  double tol = o.abs_tol, rho0 = 0.0, last = 0.0;
  int status = TPS_OK;
  do {
    fine_vmult64(h, pv, x, s);
    TPS_CUDA(launch_sub_f64(pv, b, pv, N, s));
    apply_vcycle64(h, o.precision, false, Vp(0), pv, s);
    double rho = std::sqrt(dev_dot(h, Vp(0), Vp(0), s));
    if (!std::isfinite(rho)) {
      status = TPS_ERR_NONFINITE;
      break;
    }
    if (acc == 0) {
      rho0 = rho;
      tol = std::max(o.abs_tol, o.rel_tol * rho);
      rep->initial_residual = rho;
    }
    last = rho;
    if (acc < TPS_MAX_HISTORY) rep->history[acc] = rho0 > 0 ? rho / rho0 : 0.0;
    if (rho <= tol) { state = 1; break; }
    if (acc >= o.max_iter) { state = 2; break; }
    gam.assign(basis + 1, 0.0);
    gam[0] = rho;
    TPS_CUDA(launch_scale_f64(Vp(0), 1.0 / rho, N, s));
    int dimk = 0;
    for (int inner = 0; inner < basis && state == 0 && inner + 1 < nvec; ++inner) {
      ++acc;
      fine_vmult64(h, pv, Vp(inner), s);
      apply_vcycle64(h, o.precision, false, Vp(inner + 1), pv, s);
      dimk = inner + 1;
      for (int i = 0; i < dimk; ++i) {
        hv[i] = dev_dot(h, Vp(inner + 1), Vp(i), s);
        TPS_CUDA(launch_axpy_f64(Vp(inner + 1), -hv[i], Vp(i), N, s));
      }
      const double sn = std::sqrt(dev_dot(h, Vp(inner + 1), Vp(inner + 1), s));
      hv[inner + 1] = sn;
      if (sn != 0.0) TPS_CUDA(launch_scale_f64(Vp(inner + 1), 1.0 / sn, N, s));
      for (int i = 0; i < inner; ++i) {
        const double c = ci[i], sv = si[i], d0 = hv[i];
        hv[i] = c * d0 + sv * hv[i + 1];
        hv[i + 1] = -sv * d0 + c * hv[i + 1];
      }
      const double r = 1.0 / std::sqrt(hv[inner] * hv[inner] + hv[inner + 1] * hv[inner + 1]);
      si[inner] = hv[inner + 1] * r;
      ci[inner] = hv[inner] * r;
      hv[inner] = ci[inner] * hv[inner] + si[inner] * hv[inner + 1];
      gam[inner + 1] = -si[inner] * gam[inner];
      gam[inner] *= ci[inner];
      for (int i = 0; i < dimk; ++i) H[i * basis + inner] = hv[i];
      rho = std::fabs(gam[dimk]);
      last = rho;
      if (acc < TPS_MAX_HISTORY) rep->history[acc] = rho0 > 0 ? rho / rho0 : 0.0;
      if (!std::isfinite(rho)) {
        status = TPS_ERR_NONFINITE;
        state = 2;
      } else if (rho <= tol) {
        state = 1;
      } else if (acc >= o.max_iter) {
        state = 2;
      }
    }
    std::vector<double> y(dimk, 0.0);
    for (int i = dimk - 1; i >= 0; --i) {
      double t = gam[i];
      for (int j = i + 1; j < dimk; ++j) t -= H[i * basis + j] * y[j];
      y[i] = t / H[i * basis + i];
    }
    for (int i = 0; i < dimk; ++i) TPS_CUDA(launch_axpy_f64(x, y[i], Vp(i), N, s));
  } while (state == 0 && status == TPS_OK);
  TPS_CUDA(cudaEventRecord(h->ev1, s));
  TPS_CUDA(cudaEventSynchronize(h->ev1));
  float ms = 0.f;
  TPS_CUDA(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  rep->time_ms = ms;
  rep->iterations = acc;
  rep->final_residual = rho0 > 0 ? last / rho0 : 0.0;
  rep->converged = state == 1 ? 1 : 0;
  if (status == TPS_OK && state != 1) status = TPS_ERR_NOT_CONVERGED;
  return status;
}

}  // namespace

extern "C" {

void tps_solve_opts_default(tps_solve_opts *o)
{
  if (!o) return;
  o->driver = TPS_DRIVER_CG;
  o->precision = TPS_VCYCLE_F32;
  o->symmetric = 1;
  o->max_iter = 100;
  o->rel_tol = 1e-10;
  o->abs_tol = 1e-16;
  o->use_graph = 1;
}

int tps_create(const tps_problem *pb, tps_handle **out)
{
  g_create_error.clear();
  if (!pb || !out) {
    g_create_error = "null argument";
    return TPS_ERR_INVALID;
  }
  *out = nullptr;
  std::unique_ptr<tps_handle> h;
  try {
    if (pb->dim != 2 && pb->dim != 3) throw ApiError(TPS_ERR_INVALID, "dim must be 2 or 3");
    if (pb->degree < 1 || pb->degree > kMaxDegree)
      throw ApiError(TPS_ERR_UNSUPPORTED, "degree must be in 1..7");
    if (pb->n_coarse < 2) throw ApiError(TPS_ERR_INVALID, "n_coarse must be >= 2");
    if (pb->n_levels < 1 || pb->n_levels > 12) throw ApiError(TPS_ERR_INVALID, "n_levels must be in 1..12");
    if (!(pb->relaxation > 0.0)) throw ApiError(TPS_ERR_INVALID, "relaxation must be positive");
    const int64_t nf = static_cast<int64_t>(pb->n_coarse) << (pb->n_levels - 1);
    const int64_t N1f = nf * pb->degree + 1;
    const int64_t Nf = pb->dim == 3 ? N1f * N1f * N1f : N1f * N1f;
    if (Nf >= (int64_t(1) << 31)) throw ApiError(TPS_ERR_INVALID, "finest level exceeds 2^31 DoFs");
    h.reset(new tps_handle);
    h->dim = pb->dim;
    h->k = pb->degree;
    h->n_coarse = pb->n_coarse;
    h->n_levels = pb->n_levels;
    h->omega = pb->relaxation;
    h->device = pb->device;
    TPS_CUDA(cudaSetDevice(pb->device));
    TPS_CUDA(cudaDeviceGetAttribute(&h->n_sm, cudaDevAttrMultiProcessorCount, pb->device));
    for (int l = 0; l < pb->n_levels; ++l) {
      LevelGeomH g;
      g.n = pb->n_coarse << l;
      g.N1 = g.n * pb->degree + 1;
      g.N = pb->dim == 3 ? int64_t(g.N1) * g.N1 * g.N1 : int64_t(g.N1) * g.N1;
      g.h = 1.0 / g.n;
      h->lv.push_back(g);
    }
    h->kt = kernel_table(pb->degree);
    if (!h->kt) throw ApiError(TPS_ERR_UNSUPPORTED, "degree not compiled in");
    h->D = make_degree_data(pb->degree);
    TPS_CUDA(h->kt->upload(h->D));
    if (pb->kappa) {
      h->has_kappa = true;
      set_kappa_levels(h.get(), pb->kappa);
    }
    // the single coarse patch is an exact solve only for a unit coefficient on 2 cells
    h->dense_coarse = pb->n_coarse != 2 || h->has_kappa;
    if (h->dense_coarse) {
      const int64_t m1 = int64_t(pb->n_coarse) * pb->degree - 1;
      const int64_t ni = pb->dim == 3 ? m1 * m1 * m1 : m1 * m1;
      if (ni > 4096) throw ApiError(TPS_ERR_INVALID, "coarse level too large for the dense coarse solve");
      build_dense_coarse(h.get());
    }
  } catch (const ApiError &e) {
    g_create_error = e.what();
    return e.code;
  } catch (const std::bad_alloc &) {
    g_create_error = "host allocation failed";
    return TPS_ERR_ALLOC;
  } catch (const std::exception &e) {
    g_create_error = e.what();
    return TPS_ERR_INVALID;
  }
  *out = h.release();
  return TPS_OK;
}

int tps_destroy(tps_handle *h)
{
  if (!h) return TPS_ERR_INVALID;
  cudaSetDevice(h->device);
  delete h;
  return TPS_OK;
}

const char *tps_last_error(const tps_handle *h)
{
  if (!h) return g_create_error.c_str();
  return h->err.c_str();
}

int tps_level_info(const tps_handle *h, int level, int64_t *n_dofs, int *cells_per_dim)
{
  if (!h) return TPS_ERR_INVALID;
  if (level < 0 || level >= h->n_levels) return TPS_ERR_INVALID;
  if (n_dofs) *n_dofs = h->lv[level].N;
  if (cells_per_dim) *cells_per_dim = h->lv[level].n;
  return TPS_OK;
}

int tps_laplace_vmult(tps_handle *h, int level, int dtype, void *dst, const void *src, void *stream)
{
  return guarded(h, [&] {
    check_level(h, level);
    const int p = dt_index(dtype);
    if (!dst || !src) throw ApiError(TPS_ERR_INVALID, "null vector");
    if (dst == src) throw ApiError(TPS_ERR_INVALID, "dst and src must not alias");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const LevelGeomH &g = h->lv[level];
    level_laplace(h, level, p, lex_layout(h, level), dst, src, nullptr, 0, s);
    TPS_CUDA(launch_copy_boundary(dst, src, h->dim, g.N1, p == 0 ? 8 : 4, s));
  });
}

int tps_smoother_step(tps_handle *h, int level, int dtype, void *x, const void *b, int zero_init,
                      int reverse, void *stream)
{
  return guarded(h, [&] {
    check_level(h, level);
    if (!x || !b) throw ApiError(TPS_ERR_INVALID, "null vector");
    if (x == b) throw ApiError(TPS_ERR_INVALID, "x and b must not alias");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const LevelGeomH &g = h->lv[level];
    if (dtype == TPS_TF32 || dtype == TPS_TF32X3) {
      tc_smoother_step(h, level, x, b, zero_init != 0, reverse != 0, dtype == TPS_TF32X3 ? 3 : 1, s);
      return;
    }
    const int p = dt_index(dtype);
    if (zero_init) TPS_CUDA(cudaMemsetAsync(x, 0, (p == 0 ? 8 : 4) * g.N, s));
    smoother_sweep(h, level, p, lex_layout(h, level), x, b, reverse != 0, zero_init != 0, nullptr, s);
  });
}

int tps_smoother_step_variant(tps_handle *h, int level, int dtype, void *x, const void *b, int zero_init,
                              int reverse, int variant, void *stream)
{
  if (variant == TPS_SMOOTHER_FUSED) return tps_smoother_step(h, level, dtype, x, b, zero_init, reverse, stream);
  return guarded(h, [&] {
    check_level(h, level);
    if (!x || !b) throw ApiError(TPS_ERR_INVALID, "null vector");
    if (x == b) throw ApiError(TPS_ERR_INVALID, "x and b must not alias");
    if (variant != TPS_SMOOTHER_SEPARATE && variant != TPS_SMOOTHER_GLOBAL && variant != TPS_SMOOTHER_EXACT &&
        variant != TPS_SMOOTHER_ADDITIVE)
      throw ApiError(TPS_ERR_INVALID, "unknown smoother variant");
    if (h->has_kappa)
      throw ApiError(TPS_ERR_UNSUPPORTED, "the separate-kernel smoother variants have constant coefficients");
    const int p = dt_index(dtype);
    const size_t es = p == 0 ? 8 : 4;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const LevelGeomH &g = h->lv[level];
    const VecLayout lay = lex_layout(h, level);
    if (h->var_r[p].bytes < es * h->fine().N) h->var_r[p].alloc(es * h->fine().N);
    const void *inv = nullptr;
    if (variant == TPS_SMOOTHER_EXACT) {
      if (!h->dense_inv[p].p) {
        const std::vector<double> a = dense_patch_inverse(h->D, h->dim);
        if (p == 0) {
          h->dense_inv[0].alloc(8 * a.size());
          TPS_CUDA(cudaMemcpy(h->dense_inv[0].p, a.data(), 8 * a.size(), cudaMemcpyHostToDevice));
        } else {
          const std::vector<float> f(a.begin(), a.end());
          h->dense_inv[1].alloc(4 * f.size());
          TPS_CUDA(cudaMemcpy(h->dense_inv[1].p, f.data(), 4 * f.size(), cudaMemcpyHostToDevice));
        }
      }
      inv = h->dense_inv[p].p;
    }
    if (zero_init) TPS_CUDA(cudaMemsetAsync(x, 0, es * g.N, s));
    if (variant == TPS_SMOOTHER_ADDITIVE) {
      additive_sweep(h, level, p, lay, x, b, zero_init != 0, s);
      return;
    }
    const int nc = 1 << h->dim;
    for (int i = 0; i < nc; ++i) {
      const int c = reverse ? nc - 1 - i : i;
      if (variant == TPS_SMOOTHER_GLOBAL)
        level_laplace(h, level, p, lay, h->var_r[p].p, x, b, 1, s);  // r = b - A x on interior rows
      else
        TPS_CUDA(h->kt->patch_residual[h->dim - 2][p](g, lay, x, b, h->var_r[p].p, c, s));
      TPS_CUDA(h->kt->patch_solve[h->dim - 2][p](g, lay, x, h->var_r[p].p, inv, c, h->omega, s));
    }
  });
}

int tps_prolongate_add(tps_handle *h, int to_level, int dtype, void *fine, const void *coarse,
                       void *stream)
{
  return guarded(h, [&] {
    check_level(h, to_level, 1);
    const int p = dt_index(dtype);
    if (!fine || !coarse) throw ApiError(TPS_ERR_INVALID, "null vector");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    VcycleVectors &V = vcycle_vectors(h, p);
    TPS_CUDA(h->kt->prolong[h->dim - 2][p](h->lv[to_level - 1], lex_layout(h, to_level - 1),
                                           lex_layout(h, to_level), fine, coarse,
                                           V.tmp[to_level]->p, s));
  });
}

int tps_restrict_add(tps_handle *h, int from_level, int dtype, void *coarse, const void *fine,
                     void *stream)
{
  return guarded(h, [&] {
    check_level(h, from_level, 1);
    const int p = dt_index(dtype);
    if (!fine || !coarse) throw ApiError(TPS_ERR_INVALID, "null vector");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    VcycleVectors &V = vcycle_vectors(h, p);
    TPS_CUDA(h->kt->restrict_[h->dim - 2][p](h->lv[from_level - 1], lex_layout(h, from_level - 1),
                                             lex_layout(h, from_level), coarse, fine,
                                             V.tmp[from_level]->p, 1, s));
  });
}

int tps_fmg(tps_handle *h, int precision, int n_cycles, const double *const *rhs, const double *const *bnd,
            double *x, tps_report *report, void *stream)
{
  return guarded(h, [&] {
    if (!rhs || !x) throw ApiError(TPS_ERR_INVALID, "null argument");
    if (n_cycles < 1) throw ApiError(TPS_ERR_INVALID, "n_cycles must be >= 1");
    for (int l = 0; l < h->n_levels; ++l)
      if (!rhs[l] || (bnd && !bnd[l])) throw ApiError(TPS_ERR_INVALID, "a right-hand side (or Dirichlet vector) per level is required");
    fmg(h, precision, n_cycles, rhs, bnd, x, report, static_cast<cudaStream_t>(stream));
    if (take_timeout_flag(h, static_cast<cudaStream_t>(stream))) {
      report->converged = 0;
      throw ApiError(TPS_ERR_TIMEOUT, status_message(TPS_ERR_TIMEOUT));
    }
  });
}

int tps_vcycle(tps_handle *h, int precision, int symmetric, double *dst, const double *src,
               void *stream)
{
  return guarded(h, [&] {
    if (!dst || !src) throw ApiError(TPS_ERR_INVALID, "null vector");
    apply_vcycle64(h, precision, symmetric != 0, dst, src, static_cast<cudaStream_t>(stream));
  });
}

int tps_solve(tps_handle *h, const tps_solve_opts *opts, const double *b, double *x,
              tps_report *report, void *stream)
{
  int status = TPS_OK;
  int rc = guarded(h, [&] {
    if (!opts || !b || !x || !report) throw ApiError(TPS_ERR_INVALID, "null argument");
    if (opts->max_iter < 1) throw ApiError(TPS_ERR_INVALID, "max_iter must be >= 1");
    std::memset(report, 0, sizeof(*report));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (opts->driver == TPS_DRIVER_CG)
      status = solve_cg(h, *opts, b, x, report, s);
    else if (opts->driver == TPS_DRIVER_GMRES)
      status = solve_gmres(h, *opts, b, x, report, s);
    else
      throw ApiError(TPS_ERR_INVALID, "unknown driver");
    if (take_timeout_flag(h, s)) {
      status = TPS_ERR_TIMEOUT;
      report->converged = 0;
    }
  });
  if (rc != TPS_OK) return rc;
  h->err = status_message(status);
  return status;
}

int tps_set_kappa(tps_handle *h, const double *kappa, int rebuild_coarse)
{
  return guarded(h, [&] {
    if (!h->has_kappa) throw ApiError(TPS_ERR_INVALID, "the handle was created with kappa = NULL");
    if (!kappa) throw ApiError(TPS_ERR_INVALID, "null kappa");
    TPS_CUDA(cudaDeviceSynchronize());
    set_kappa_levels(h, kappa);
    if (rebuild_coarse) {
      build_dense_coarse(h);
      for (int p = 0; p < 2; ++p) {
        VcycleVectors &V = h->vc[p];
        if (!V.ready) continue;
        const size_t n2 = h->coarse_inv_host.size();
        if (p == 0) {
          TPS_CUDA(cudaMemcpy(V.coarse_inv.p, h->coarse_inv_host.data(), 8 * n2, cudaMemcpyHostToDevice));
        } else {
          std::vector<float> f(h->coarse_inv_host.begin(), h->coarse_inv_host.end());
          TPS_CUDA(cudaMemcpy(V.coarse_inv.p, f.data(), 4 * n2, cudaMemcpyHostToDevice));
        }
      }
    }
    if (h->graph) {  // re-captured on the next solve
      cudaGraphExecDestroy(h->graph);
      h->graph = nullptr;
    }
  });
}

int tps_mass_vmult(tps_handle *h, double *dst, const double *src, void *stream)
{
  return guarded(h, [&] {
    if (!dst || !src || dst == src) throw ApiError(TPS_ERR_INVALID, "bad vectors");
    const int L = h->n_levels - 1;
    TPS_CUDA(h->kt->mass[h->dim - 2](h->lv[L], lex_layout(h, L), dst, src,
                                     static_cast<cudaStream_t>(stream)));
  });
}

int tps_assemble_rhs(tps_handle *h, int level, const double *f_quad, double *b, void *stream)
{
  return guarded(h, [&] {
    check_level(h, level);
    if (!f_quad || !b) throw ApiError(TPS_ERR_INVALID, "null vector");
    TPS_CUDA(h->kt->assemble_rhs[h->dim - 2](h->lv[level], lex_layout(h, level), b, f_quad,
                                             static_cast<cudaStream_t>(stream)));
  });
}

int tps_adjoint(tps_handle *h, const tps_solve_opts *opts, const double *u, const double *g, double *dJdf,
                double *dJdkappa, tps_report *report, void *stream)
{
  int status = TPS_OK;
  int rc = guarded(h, [&] {
    if (!opts || !u || !g || !dJdf || !report) throw ApiError(TPS_ERR_INVALID, "null argument");
    if (opts->driver != TPS_DRIVER_CG) throw ApiError(TPS_ERR_INVALID, "the adjoint solve uses the CG driver");
    if (opts->max_iter < 1) throw ApiError(TPS_ERR_INVALID, "max_iter must be >= 1");
    if (dJdkappa && !h->has_kappa) throw ApiError(TPS_ERR_INVALID, "dJ/dkappa needs a handle created with kappa");
    if (dJdf == g || dJdf == u) throw ApiError(TPS_ERR_INVALID, "dJ/df must not alias u or g");
    std::memset(report, 0, sizeof(*report));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int L = h->n_levels - 1;
    const LevelGeomH &gf = h->fine();
    const int64_t N = gf.N;
    if (!h->adj_g.p) h->adj_g.alloc(sizeof(double) * N);
    if (!h->adj_lam.p) h->adj_lam.alloc(sizeof(double) * N);
    double *gb = h->adj_g.as<double>(), *lam = h->adj_lam.as<double>();
    // adjoint right-hand side: g with its Dirichlet rows zeroed, so lambda = 0 there
    TPS_CUDA(cudaMemsetAsync(lam, 0, sizeof(double) * N, s));
    TPS_CUDA(cudaMemcpyAsync(gb, g, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
    TPS_CUDA(launch_copy_boundary(gb, lam, h->dim, gf.N1, 8, s));
    status = solve_cg(h, *opts, gb, lam, report, s);
    TPS_CUDA(h->kt->mass[h->dim - 2](gf, lex_layout(h, L), dJdf, lam, s));
    if (dJdkappa) {
      TPS_CUDA(h->kt->cell_energy[h->dim - 2](gf, lex_layout(h, L), dJdkappa, u, lam, s));
      const int64_t nc = h->dim == 3 ? int64_t(gf.n) * gf.n * gf.n : int64_t(gf.n) * gf.n;
      TPS_CUDA(launch_scale_f64(dJdkappa, -1.0, nc, s));
    }
    if (take_timeout_flag(h, s)) {
      status = TPS_ERR_TIMEOUT;
      report->converged = 0;
    }
  });
  if (rc != TPS_OK) return rc;
  h->err = status_message(status);
  return status;
}

int tps_cell_energy(tps_handle *h, const double *u, const double *lam, double *energy, void *stream)
{
  return guarded(h, [&] {
    if (!u || !lam || !energy) throw ApiError(TPS_ERR_INVALID, "null vector");
    const int L = h->n_levels - 1;
    TPS_CUDA(h->kt->cell_energy[h->dim - 2](h->lv[L], lex_layout(h, L), energy, u, lam,
                                            static_cast<cudaStream_t>(stream)));
  });
}

int tps_smoother_variants(tps_handle *h, int dtype, int *ppb)
{
  return guarded(h, [&] {
    const int p = dt_index(dtype);
    if (!ppb) throw ApiError(TPS_ERR_INVALID, "null output");
    for (int v = 0; v < kSmootherVariants; ++v) ppb[v] = h->kt->smoother_ppb(h->dim, p == 0 ? 0 : 1, v);
  });
}

int tps_set_smoother_variant(tps_handle *h, int dtype, int level, int variant)
{
  return guarded(h, [&] {
    const int p = dt_index(dtype);
    check_level(h, level);
    if (variant < 0 || variant >= kSmootherVariants) throw ApiError(TPS_ERR_INVALID, "variant out of range");
    if (static_cast<int>(h->sm_variant[p].size()) != h->n_levels) h->sm_variant[p].assign(h->n_levels, 0);
    h->sm_variant[p][level] = variant;
    if (h->graph) {  // later solves re-capture with the chosen kernel
      cudaGraphExecDestroy(h->graph);
      h->graph = nullptr;
    }
  });
}

int tps_set_smoother_kind(tps_handle *h, int kind, double damping)
{
  return guarded(h, [&] {
    if (kind != TPS_SMOOTHER_FUSED && kind != TPS_SMOOTHER_ADDITIVE)
      throw ApiError(TPS_ERR_INVALID, "kind must be TPS_SMOOTHER_FUSED or TPS_SMOOTHER_ADDITIVE");
    if (kind == TPS_SMOOTHER_ADDITIVE) {
      if (h->has_kappa) throw ApiError(TPS_ERR_UNSUPPORTED, "the additive step has a constant coefficient");
      if (!(damping >= 0.0 && damping < 2.0 / (1 << h->dim)))
        throw ApiError(TPS_ERR_INVALID, "additive damping must lie in [0, 2/2^dim) (0: 1/2^dim)");
      h->add_omega = damping;
      ensure_additive_scratch(h, 0);
      ensure_additive_scratch(h, 1);
    }
    h->sm_kind = kind;
    if (h->graph) {  // a captured CG iteration holds the previous smoothing
      cudaGraphExecDestroy(h->graph);
      h->graph = nullptr;
    }
  });
}

int tps_get_smoother_variant(tps_handle *h, int dtype, int level, int *variant)
{
  return guarded(h, [&] {
    const int p = dt_index(dtype);
    check_level(h, level);
    if (!variant) throw ApiError(TPS_ERR_INVALID, "null output");
    *variant = level < static_cast<int>(h->sm_variant[p].size()) ? h->sm_variant[p][level]
                                                                 : default_variant(h, level, p);
  });
}

int tps_set_operator_layers(tps_handle *h, int dtype, int level, int layers)
{
  return guarded(h, [&] {
    const int p = dt_index(dtype);
    check_level(h, level);
    if (layers != 0 && layers != 1 && layers != 2 && layers != 4 && layers != 8 && layers != 16)
      throw ApiError(TPS_ERR_INVALID, "operator layers must be 0 (default), 1, 2, 4, 8 or 16");
    if (static_cast<int>(h->op_layers[p].size()) != h->n_levels) h->op_layers[p].assign(h->n_levels, 0);
    h->op_layers[p][level] = layers;
    if (h->graph) {  // later solves re-capture with the chosen tile depth
      cudaGraphExecDestroy(h->graph);
      h->graph = nullptr;
    }
  });
}

int tps_get_operator_layers(tps_handle *h, int dtype, int level, int *layers)
{
  return guarded(h, [&] {
    const int p = dt_index(dtype);
    check_level(h, level);
    if (!layers) throw ApiError(TPS_ERR_INVALID, "null output");
    *layers = level < static_cast<int>(h->op_layers[p].size()) ? h->op_layers[p][level] : 0;
  });
}

int tps_autotune(tps_handle *h, int dtype, int *ppb_per_level)
{
  return guarded(h, [&] {
    const int p = dt_index(dtype);
    if (!h->own_stream) TPS_CUDA(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
    autotune_levels(h, p, h->own_stream);
    TPS_CUDA(cudaStreamSynchronize(h->own_stream));
    if (h->graph) {  // later solves re-capture with the chosen kernels
      cudaGraphExecDestroy(h->graph);
      h->graph = nullptr;
    }
    if (ppb_per_level)
      for (int l = 0; l < h->n_levels; ++l)
        ppb_per_level[l] = h->kt->smoother_ppb(h->dim, p == 0 ? 0 : 1, h->sm_variant[p][l]);
  });
}

int tps_time_smoother(tps_handle *h, int level, int dtype, int sweeps, double *ms_per_sweep,
                      void *stream)
{
  return guarded(h, [&] {
    check_level(h, level);
    const bool tc = dtype == TPS_TF32 || dtype == TPS_TF32X3;
    if (tc) check_tc(h, dtype == TPS_TF32X3 ? 3 : 1);
    if (dtype == TPS_TF32X3 && h->k != 4)
      throw ApiError(TPS_ERR_UNSUPPORTED, "the three-term TF32 tensor-core smoother needs degree 4");
    const int p = tc ? 1 : dt_index(dtype);
    if (sweeps < 1 || !ms_per_sweep) throw ApiError(TPS_ERR_INVALID, "sweeps >= 1 and an output are required");
    ensure_krylov(h);
    VcycleVectors &V = vcycle_vectors(h, p);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    TPS_CUDA(cudaEventRecord(h->ev0, s));
    for (int i = 0; i < sweeps; ++i)
      smoother_sweep(h, level, p, V.layout[level], V.su[level]->p, V.d[level]->p, false, false,
                     &V.maps[level], s, tc);
    TPS_CUDA(cudaEventRecord(h->ev1, s));
    TPS_CUDA(cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    TPS_CUDA(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    *ms_per_sweep = ms / sweeps;
    if (take_timeout_flag(h, s)) throw ApiError(TPS_ERR_TIMEOUT, status_message(TPS_ERR_TIMEOUT));
  });
}

int tps_solve_host(tps_handle *h, const tps_solve_opts *opts, const double *b_host, double *x_host,
                   tps_report *report)
{
  return tps_solve_host_guess(h, opts, b_host, x_host, x_host, report);
}

int tps_solve_host_guess(tps_handle *h, const tps_solve_opts *opts, const double *b_host, const double *x0_host,
                         double *x_host, tps_report *report)
{
  if (!h) return TPS_ERR_INVALID;
  if (!b_host || !x_host) {
    h->err = "null host buffer";
    return TPS_ERR_INVALID;
  }
  int status = TPS_OK;
  int rc = guarded(h, [&] {
    const int64_t N = h->fine().N;
    if (!h->own_stream) TPS_CUDA(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
    cudaStream_t s = h->own_stream;
    if (!h->host_b.p) h->host_b.alloc(sizeof(double) * N);
    if (!h->host_x.p) h->host_x.alloc(sizeof(double) * N);
    TPS_CUDA(cudaMemcpyAsync(h->host_b.p, b_host, sizeof(double) * N, cudaMemcpyHostToDevice, s));
    if (x0_host)
      TPS_CUDA(cudaMemcpyAsync(h->host_x.p, x0_host, sizeof(double) * N, cudaMemcpyHostToDevice, s));
    else
      TPS_CUDA(cudaMemsetAsync(h->host_x.p, 0, sizeof(double) * N, s));
    status = tps_solve(h, opts, h->host_b.as<double>(), h->host_x.as<double>(), report, s);
    if (status == TPS_OK || status == TPS_ERR_NOT_CONVERGED) {
      TPS_CUDA(cudaMemcpyAsync(x_host, h->host_x.p, sizeof(double) * N, cudaMemcpyDeviceToHost, s));
      TPS_CUDA(cudaStreamSynchronize(s));
    }
  });
  if (rc != TPS_OK) return rc;
  h->err = status_message(status);  // the message of the inner tps_solve
  return status;
}

int tps_solve_host_many(tps_handle *h, const tps_solve_opts *opts, int n, const double *const *b_host,
                        double *const *x_host, tps_report *reports)
{
  if (!h) return TPS_ERR_INVALID;
  if (!opts || n < 1 || !b_host || !x_host || !reports) {
    h->err = "null argument or n < 1";
    return TPS_ERR_INVALID;
  }
  for (int i = 0; i < n; ++i)
    if (!b_host[i] || !x_host[i]) {
      h->err = "null host buffer";
      return TPS_ERR_INVALID;
    }
  int status = TPS_OK;
  const int rc = guarded(h, [&] {
    const int64_t N = h->fine().N;
    const size_t bytes = sizeof(double) * N;
    if (!h->own_stream) TPS_CUDA(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
    if (!h->copy_stream) TPS_CUDA(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
    for (int i = 0; i < 2; ++i) {
      if (!h->pipe_b[i].p) h->pipe_b[i].alloc(bytes);
      if (!h->pipe_x[i].p) h->pipe_x[i].alloc(bytes);
      if (!h->pipe_in[i]) TPS_CUDA(cudaEventCreateWithFlags(&h->pipe_in[i], cudaEventDisableTiming));
      if (!h->pipe_done[i]) TPS_CUDA(cudaEventCreateWithFlags(&h->pipe_done[i], cudaEventDisableTiming));
      if (!h->pipe_out[i]) TPS_CUDA(cudaEventCreateWithFlags(&h->pipe_out[i], cudaEventDisableTiming));
    }
    if (!h->host_x.p) h->host_x.alloc(bytes);
    cudaStream_t s = h->own_stream, cs = h->copy_stream;
    // the copies stay ordered on the copy stream: H2D of b[i+1] is queued while
    // solve i runs, then D2H of x[i] once solve i is done, so both overlap solve
    // i+1.  Every solve starts from zero in host_x (a fixed vector, so the
    // captured CG iteration is reused) and is copied out to pipe_x.
    try {
      TPS_CUDA(cudaMemcpyAsync(h->pipe_b[0].p, b_host[0], bytes, cudaMemcpyHostToDevice, cs));
      TPS_CUDA(cudaEventRecord(h->pipe_in[0], cs));
      for (int i = 0; i < n; ++i) {
        const int sl = i & 1;
        if (i + 1 < n) {  // pipe_b[sl ^ 1] was last read by solve i-1, which has returned
          TPS_CUDA(cudaMemcpyAsync(h->pipe_b[sl ^ 1].p, b_host[i + 1], bytes, cudaMemcpyHostToDevice, cs));
          TPS_CUDA(cudaEventRecord(h->pipe_in[sl ^ 1], cs));
        }
        TPS_CUDA(cudaStreamWaitEvent(s, h->pipe_in[sl], 0));
        TPS_CUDA(cudaMemsetAsync(h->host_x.p, 0, bytes, s));
        const int si = tps_solve(h, opts, h->pipe_b[sl].as<double>(), h->host_x.as<double>(), &reports[i], s);
        if (si != TPS_OK && si != TPS_ERR_NOT_CONVERGED && si != TPS_ERR_BREAKDOWN && si != TPS_ERR_NONFINITE &&
            si != TPS_ERR_TIMEOUT)
          throw ApiError(si, h->err);
        if (si != TPS_OK && (status == TPS_OK || status == TPS_ERR_NOT_CONVERGED)) status = si;
        if (si == TPS_OK || si == TPS_ERR_NOT_CONVERGED) {
          // pipe_x[sl] still holds x[i-2] until its D2H has completed
          if (i >= 2) TPS_CUDA(cudaStreamWaitEvent(s, h->pipe_out[sl], 0));
          TPS_CUDA(cudaMemcpyAsync(h->pipe_x[sl].p, h->host_x.p, bytes, cudaMemcpyDeviceToDevice, s));
          TPS_CUDA(cudaEventRecord(h->pipe_done[sl], s));
          TPS_CUDA(cudaStreamWaitEvent(cs, h->pipe_done[sl], 0));
          TPS_CUDA(cudaMemcpyAsync(x_host[i], h->pipe_x[sl].p, bytes, cudaMemcpyDeviceToHost, cs));
          TPS_CUDA(cudaEventRecord(h->pipe_out[sl], cs));
        } else {
          // no result to copy: later solves must not wait on a stale event
          TPS_CUDA(cudaEventRecord(h->pipe_out[sl], cs));
        }
      }
      TPS_CUDA(cudaStreamSynchronize(cs));
    } catch (...) {
      // no copy may still be writing into the caller's buffers after the return
      cudaStreamSynchronize(cs);
      cudaStreamSynchronize(s);
      throw;
    }
  });
  if (rc != TPS_OK) return rc;
  h->err = status_message(status);
  return status;
}

int tps_check_colouring(int dim, int degree, int n_cells)
{
  g_create_error.clear();
  if ((dim != 2 && dim != 3) || degree < 1 || degree > kMaxDegree || n_cells < 2 || n_cells > 512) {
    g_create_error = "tps_check_colouring: dim 2 or 3, degree 1..7, 2..512 cells";
    return TPS_ERR_INVALID;
  }
  const int k = degree, n = n_cells, N1 = n * k + 1, nc = 1 << dim;
  const int64_t NN = dim == 3 ? int64_t(N1) * N1 * N1 : int64_t(N1) * N1;
  auto at = [&](int x, int y, int z) { return x + int64_t(N1) * (y + int64_t(N1) * z); };
  std::vector<uint8_t> interior(static_cast<size_t>(NN));  // owner marks of the current colour
  std::vector<uint8_t> centre(static_cast<size_t>(NN), 0);  // vertex patches seen over all colours
  int64_t total = 0;
  auto fail = [&](const std::string &m) {
    g_create_error = "tps_check_colouring: " + m;
    return TPS_ERR_INVALID;
  };
  for (int c = 0; c < nc; ++c) {
    int nx, ny, nz, count;
    colour_lattice(dim, n, c, nx, ny, nz, count);
    total += count;
    std::fill(interior.begin(), interior.end(), 0);
    const int cx = c & 1, cy = (c >> 1) & 1, cz = (c >> 2) & 1;
    const int ez = dim == 3 ? 2 * k - 1 : 1;  // interior extent in z
    // the interiors of one colour's patches are disjoint
    for (int jz = 0; jz < nz; ++jz)
      for (int jy = 0; jy < ny; ++jy)
        for (int jx = 0; jx < nx; ++jx) {
          const int fx = (cx + 2 * jx) * k, fy = (cy + 2 * jy) * k, fz = dim == 3 ? (cz + 2 * jz) * k : -1;
          if (fx + 2 * k > N1 - 1 || fy + 2 * k > N1 - 1 || (dim == 3 && fz + 2 * k > N1 - 1))
            return fail("patch box outside the level");
          const int64_t v = at(fx + k, fy + k, dim == 3 ? fz + k : 0);
          if (centre[v]) return fail("vertex patch of colour " + std::to_string(c) + " seen twice");
          centre[v] = 1;
          for (int z = 0; z < ez; ++z)
            for (int y = 1; y < 2 * k; ++y)
              for (int x = 1; x < 2 * k; ++x) {
                const int64_t i = at(fx + x, fy + y, dim == 3 ? fz + 1 + z : 0);
                if (interior[i]) return fail("colour " + std::to_string(c) + ": patch interiors overlap");
                interior[i] = 1;
              }
        }
    // no patch reads (its box ring) what another patch of the colour writes
    for (int jz = 0; jz < nz; ++jz)
      for (int jy = 0; jy < ny; ++jy)
        for (int jx = 0; jx < nx; ++jx) {
          const int fx = (cx + 2 * jx) * k, fy = (cy + 2 * jy) * k, fz = dim == 3 ? (cz + 2 * jz) * k : 0;
          const int bz = dim == 3 ? 2 * k + 1 : 1;
          for (int z = 0; z < bz; ++z)
            for (int y = 0; y <= 2 * k; ++y)
              for (int x = 0; x <= 2 * k; ++x) {
                const bool ring = x == 0 || x == 2 * k || y == 0 || y == 2 * k || (dim == 3 && (z == 0 || z == 2 * k));
                if (ring && interior[at(fx + x, fy + y, fz + z)])
                  return fail("colour " + std::to_string(c) + ": a box ring meets another patch's interior");
              }
        }
  }
  // every interior vertex is the centre of exactly one patch
  const int64_t expect = dim == 3 ? int64_t(n - 1) * (n - 1) * (n - 1) : int64_t(n - 1) * (n - 1);
  if (total != expect) return fail("patch count " + std::to_string(total) + " != " + std::to_string(expect));
  return TPS_OK;
}

int tps_device_status(tps_handle *h)
{
  bool timed_out = false;
  const int rc = guarded(h, [&] {
    TPS_CUDA(cudaDeviceSynchronize());
    timed_out = take_timeout_flag(h, nullptr);
  });
  if (rc != TPS_OK) return rc;
  if (!timed_out) return TPS_OK;
  h->err = status_message(TPS_ERR_TIMEOUT);
  return TPS_ERR_TIMEOUT;
}

int tps_selftest_wait_timeout(tps_handle *h, long long cycles, void *stream)
{
  return guarded(h, [&] {
    if (cycles < 1 || cycles > (1ll << 31)) throw ApiError(TPS_ERR_INVALID, "cycles must be in 1..2^31");
    if (!h->err_flag.p) h->err_flag.alloc(sizeof(int));
    TPS_CUDA(launch_wait_timeout_selftest(h->err_flag.as<int>(), cycles, static_cast<cudaStream_t>(stream)));
  });
}

void tps_inject_alloc_failure(int n) { g_alloc_fault.store(n > 0 ? n : 0); }

}  // extern "C"

// ---- batched solves ---------------------------------------------------------
// n independent systems (own hierarchy and work vectors each) solved by one
// CUDA graph: fork -> initial residual of every system -> join -> check ->
// while (some system active) { select -> [if active_i: one CG iteration of
// system i] on parallel branches -> check }.  The loop runs on the device;
// the host waits once at the end.

namespace {
constexpr int kMaxBatch = kBatchMax;
}  // namespace

struct tps_batch {
  std::vector<tps_handle *> sys;
  int device = 0;
  std::string err;
  std::vector<cudaStream_t> fork, body;  // capture branches (init, loop body)
  cudaStream_t aux = nullptr, own = nullptr;
  std::vector<cudaEvent_t> ev;  // fork/join events
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  cudaGraphExec_t exec = nullptr;
  // what the instantiated graph was built for
  int k_prec = -1, k_sym = -1, k_max = -1;
  double k_tol = -1.0;
  cudaStream_t k_stream = nullptr;
  std::vector<const double *> k_b;
  std::vector<double *> k_x;
  DevBuf sc_ptrs, iters, active, bnorm, hist;

  ~tps_batch()
  {
    if (exec) cudaGraphExecDestroy(exec);
    for (cudaStream_t s : fork) cudaStreamDestroy(s);
    for (cudaStream_t s : body) cudaStreamDestroy(s);
    if (aux) cudaStreamDestroy(aux);
    if (own) cudaStreamDestroy(own);
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    for (tps_handle *h : sys) tps_destroy(h);
  }
};

namespace tps {
namespace {

// x_b = b_b, r = b - A x, d = r in the V-cycle precision, rr and bb; p = q = 0
// and zero scalars, so the first loop iteration is the first CG direction
void batch_init_system(tps_handle *h, int prec, const double *b, double *x, cudaStream_t s)
{
  const int p = vprec_index(prec), L = h->n_levels - 1;
  const int64_t N = h->fine().N;
  VcycleVectors &V = h->vc[p];
  CGScalars *sc = h->scalars.as<CGScalars>();
  TPS_CUDA(cudaMemsetAsync(sc, 0, sizeof(CGScalars), s));
  TPS_CUDA(cudaMemsetAsync(h->p.p, 0, sizeof(double) * N, s));
  TPS_CUDA(cudaMemsetAsync(h->q.p, 0, sizeof(double) * N, s));
  TPS_CUDA(cudaMemsetAsync(h->r.p, 0, sizeof(double) * N, s));
  TPS_CUDA(launch_copy_boundary(x, b, h->dim, h->fine().N1, 8, s));
  level_laplace(h, L, 0, lex_layout(h, L), h->r.p, x, b, 1, s);
  TPS_CUDA(launch_cg_init(h->r.as<double>(), b, V.d[L]->p, input_kind(prec), fine_padmap(h, p), N,
                          h->partial.as<double>(), s));
  TPS_CUDA(launch_cg_finalize_init(h->partial.as<double>(), sc, s));
}

struct CaptureGuard {  // ends a capture left open by an exception
  cudaStream_t s;
  bool open = true;
  ~CaptureGuard()
  {
    if (open) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(s, &g);
      if (g) cudaGraphDestroy(g);
    }
  }
};

std::vector<cudaGraphNode_t> capture_deps(cudaStream_t s, cudaGraph_t *g)
{
  cudaStreamCaptureStatus st;
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  TPS_CUDA(cudaStreamGetCaptureInfo(s, &st, nullptr, g, &deps, &nd));
  if (st != cudaStreamCaptureStatusActive) throw ApiError(TPS_ERR_CUDA, "stream is not capturing");
  return std::vector<cudaGraphNode_t>(deps, deps + nd);
}

void batch_build(tps_batch *B, const tps_solve_opts &o, const double *const *b, double *const *x, cudaStream_t s)
{
  const int n = static_cast<int>(B->sys.size());
  const int p = vprec_index(o.precision);
  const bool sym = o.symmetric != 0;
  for (tps_handle *h : B->sys) {  // every allocation happens before the capture
    vcycle_vectors(h, p);
    ensure_krylov(h);
  }
  // autotuning (smoother variants, operator tile depth), once per distinct
  // hierarchy of the batch
  for (int i = 0; i < n; ++i) {
    tps_handle *h = B->sys[i];
    if (static_cast<int>(h->sm_variant[p].size()) == h->n_levels) continue;
    int j = 0;
    for (; j < i; ++j) {
      const tps_handle *o2 = B->sys[j];
      if (o2->dim == h->dim && o2->k == h->k && o2->n_coarse == h->n_coarse && o2->n_levels == h->n_levels &&
          static_cast<int>(o2->sm_variant[p].size()) == o2->n_levels)
        break;
    }
    if (j < i) {
      h->sm_variant[p] = B->sys[j]->sm_variant[p];
      h->op_layers[p] = B->sys[j]->op_layers[p];
    } else
      autotune_levels(h, p, s);
  }
  std::vector<CGScalars *> scp(n);
  for (int i = 0; i < n; ++i) scp[i] = B->sys[i]->scalars.as<CGScalars>();
  TPS_CUDA(cudaMemcpy(B->sc_ptrs.p, scp.data(), sizeof(CGScalars *) * n, cudaMemcpyHostToDevice));
  BatchLoop bl{B->sc_ptrs.as<CGScalars *>(), B->iters.as<int>(), B->active.as<int>(), B->bnorm.as<double>(),
               B->hist.as<double>(), n, TPS_MAX_HISTORY, o.max_iter, o.rel_tol};
  if (B->exec) {
    cudaGraphExecDestroy(B->exec);
    B->exec = nullptr;
  }
  TPS_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  CaptureGuard top{s};
  TPS_CUDA(cudaEventRecord(B->ev[n], s));
  for (int i = 0; i < n; ++i) {
    TPS_CUDA(cudaStreamWaitEvent(B->fork[i], B->ev[n], 0));
    batch_init_system(B->sys[i], o.precision, b[i], x[i], B->fork[i]);
    TPS_CUDA(cudaEventRecord(B->ev[i], B->fork[i]));
    TPS_CUDA(cudaStreamWaitEvent(s, B->ev[i], 0));
  }
  cudaGraph_t cg = nullptr;
  capture_deps(s, &cg);
  cudaGraphConditionalHandle loop;
  TPS_CUDA(cudaGraphConditionalHandleCreate(&loop, cg, 0, 0));
  TPS_CUDA(launch_batch_check(bl, 1, loop, s));
  std::vector<cudaGraphNode_t> deps = capture_deps(s, &cg);
  cudaGraphNodeParams wp{};
  wp.type = cudaGraphNodeTypeConditional;
  wp.conditional.handle = loop;
  wp.conditional.type = cudaGraphCondTypeWhile;
  wp.conditional.size = 1;
  cudaGraphNode_t wnode;
  TPS_CUDA(cudaGraphAddNode(&wnode, cg, deps.data(), deps.size(), &wp));
  cudaGraph_t bodyg = wp.conditional.phGraph_out[0];
  {
    TPS_CUDA(cudaStreamBeginCaptureToGraph(B->aux, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    CaptureGuard bg{B->aux};
    BatchConds ca{};
    for (int i = 0; i < n; ++i) TPS_CUDA(cudaGraphConditionalHandleCreate(&ca.h[i], bodyg, 0, 0));
    TPS_CUDA(launch_batch_select(B->active.as<int>(), ca, n, B->aux));
    cudaGraph_t bg_graph = nullptr;
    std::vector<cudaGraphNode_t> sel = capture_deps(B->aux, &bg_graph);
    std::vector<cudaGraphNode_t> ifn(n);
    for (int i = 0; i < n; ++i) {
      cudaGraphNodeParams ip{};
      ip.type = cudaGraphNodeTypeConditional;
      ip.conditional.handle = ca.h[i];
      ip.conditional.type = cudaGraphCondTypeIf;
      ip.conditional.size = 1;
      TPS_CUDA(cudaGraphAddNode(&ifn[i], bg_graph, sel.data(), sel.size(), &ip));
      TPS_CUDA(cudaStreamBeginCaptureToGraph(B->body[i], ip.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                             cudaStreamCaptureModeThreadLocal));
      CaptureGuard ig{B->body[i]};
      cg_iteration_body(B->sys[i], o.precision, sym, x[i], B->body[i]);
      cudaGraph_t tmp = nullptr;
      ig.open = false;
      TPS_CUDA(cudaStreamEndCapture(B->body[i], &tmp));
    }
    TPS_CUDA(cudaStreamUpdateCaptureDependencies(B->aux, ifn.data(), ifn.size(), cudaStreamSetCaptureDependencies));
    TPS_CUDA(launch_batch_check(bl, 0, loop, B->aux));
    cudaGraph_t tmp = nullptr;
    bg.open = false;
    TPS_CUDA(cudaStreamEndCapture(B->aux, &tmp));
  }
  TPS_CUDA(cudaStreamUpdateCaptureDependencies(s, &wnode, 1, cudaStreamSetCaptureDependencies));
  cudaGraph_t g = nullptr;
  top.open = false;
  TPS_CUDA(cudaStreamEndCapture(s, &g));
  cudaError_t e = cudaGraphInstantiate(&B->exec, g, 0);
  cudaGraphDestroy(g);
  TPS_CUDA(e);
  B->k_prec = o.precision;
  B->k_sym = o.symmetric != 0;
  B->k_max = o.max_iter;
  B->k_tol = o.rel_tol;
  B->k_stream = s;
  B->k_b.assign(b, b + n);
  B->k_x.assign(x, x + n);
}

template <typename F>
int batch_guarded(tps_batch *B, F &&f)
{
  if (!B) return TPS_ERR_INVALID;
  try {
    cudaError_t e = cudaSetDevice(B->device);
    if (e != cudaSuccess) throw ApiError(TPS_ERR_CUDA, cudaGetErrorString(e));
    int st = f();
    B->err = status_message(st);
    return st;
  } catch (const ApiError &e) {
    B->err = e.what();
    return e.code;
  } catch (const std::bad_alloc &) {
    B->err = "host allocation failed";
    return TPS_ERR_ALLOC;
  } catch (const std::exception &e) {
    B->err = e.what();
    return TPS_ERR_INVALID;
  }
}

}  // namespace
}  // namespace tps

extern "C" {

int tps_batch_create(const tps_problem *problems, int n_systems, tps_batch **out)
{
  if (!problems || !out || n_systems < 1 || n_systems > kMaxBatch) {
    g_create_error = "tps_batch_create: 1..256 problems and an output pointer are required";
    return TPS_ERR_INVALID;
  }
  *out = nullptr;
  tps_batch *B = nullptr;
  try {
    B = new tps_batch;
  } catch (const std::bad_alloc &) {
    return TPS_ERR_ALLOC;
  }
  B->device = problems[0].device;
  for (int i = 0; i < n_systems; ++i) {
    if (problems[i].device != B->device) {
      g_create_error = "tps_batch_create: all systems must be on one device";
      delete B;
      return TPS_ERR_INVALID;
    }
    tps_handle *h = nullptr;
    const int st = tps_create(&problems[i], &h);
    if (st != TPS_OK) {
      delete B;
      return st;
    }
    B->sys.push_back(h);
  }
  const int rc = batch_guarded(B, [&] {
    const int n = n_systems;
    B->fork.resize(n);
    B->body.resize(n);
    for (int i = 0; i < n; ++i) {
      TPS_CUDA(cudaStreamCreateWithFlags(&B->fork[i], cudaStreamNonBlocking));
      TPS_CUDA(cudaStreamCreateWithFlags(&B->body[i], cudaStreamNonBlocking));
    }
    TPS_CUDA(cudaStreamCreateWithFlags(&B->aux, cudaStreamNonBlocking));
    B->ev.resize(n + 1);
    for (auto &e : B->ev) TPS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    TPS_CUDA(cudaEventCreate(&B->t0));
    TPS_CUDA(cudaEventCreate(&B->t1));
    B->sc_ptrs.alloc(sizeof(CGScalars *) * n);
    B->iters.alloc(sizeof(int) * n);
    B->active.alloc(sizeof(int) * n);
    B->bnorm.alloc(sizeof(double) * n);
    B->hist.alloc(sizeof(double) * n * TPS_MAX_HISTORY);
    return TPS_OK;
  });
  if (rc != TPS_OK) {
    g_create_error = B->err;
    delete B;
    return rc;
  }
  *out = B;
  return TPS_OK;
}

int tps_batch_destroy(tps_batch *b)
{
  if (!b) return TPS_ERR_INVALID;
  cudaSetDevice(b->device);
  delete b;
  return TPS_OK;
}

const char *tps_batch_last_error(const tps_batch *b) { return b ? b->err.c_str() : g_create_error.c_str(); }

int tps_batch_system(tps_batch *b, int i, tps_handle **h)
{
  if (!b || !h || i < 0 || i >= static_cast<int>(b->sys.size())) return TPS_ERR_INVALID;
  *h = b->sys[i];
  return TPS_OK;
}

int tps_batch_solve(tps_batch *B, const tps_solve_opts *opts, const double *const *rhs, double *const *x,
                    tps_report *reports, void *stream)
{
  TPS_RANGE("tps_batch_solve");
  return batch_guarded(B, [&]() -> int {
    if (!opts || !rhs || !x || !reports) throw ApiError(TPS_ERR_INVALID, "null argument");
    if (opts->driver != TPS_DRIVER_CG) throw ApiError(TPS_ERR_INVALID, "batched solves use the CG driver");
    if (opts->max_iter < 1) throw ApiError(TPS_ERR_INVALID, "max_iter must be >= 1");
    const int n = static_cast<int>(B->sys.size());
    for (int i = 0; i < n; ++i) {
      if (!rhs[i] || !x[i]) throw ApiError(TPS_ERR_INVALID, "null vector");
      if (vprec_tc(opts->precision)) check_tc(B->sys[i], vprec_passes(opts->precision));
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!s) {  // capture needs a non-default stream
      if (!B->own) TPS_CUDA(cudaStreamCreateWithFlags(&B->own, cudaStreamNonBlocking));
      s = B->own;
    }
    const bool same = B->exec && B->k_prec == opts->precision && B->k_sym == (opts->symmetric != 0) &&
                      B->k_max == opts->max_iter && B->k_tol == opts->rel_tol && B->k_stream == s &&
                      std::equal(B->k_b.begin(), B->k_b.end(), rhs) && std::equal(B->k_x.begin(), B->k_x.end(), x);
    if (!same) batch_build(B, *opts, rhs, x, s);
    TPS_CUDA(cudaEventRecord(B->t0, s));
    TPS_CUDA(cudaGraphLaunch(B->exec, s));
    TPS_CUDA(cudaEventRecord(B->t1, s));
    TPS_CUDA(cudaEventSynchronize(B->t1));
    float ms = 0.f;
    TPS_CUDA(cudaEventElapsedTime(&ms, B->t0, B->t1));
    std::vector<int> it(n), act(n);
    std::vector<double> bn(n), hist(static_cast<size_t>(n) * TPS_MAX_HISTORY);
    TPS_CUDA(cudaMemcpy(it.data(), B->iters.p, sizeof(int) * n, cudaMemcpyDeviceToHost));
    TPS_CUDA(cudaMemcpy(act.data(), B->active.p, sizeof(int) * n, cudaMemcpyDeviceToHost));
    TPS_CUDA(cudaMemcpy(bn.data(), B->bnorm.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
    TPS_CUDA(cudaMemcpy(hist.data(), B->hist.p, sizeof(double) * hist.size(), cudaMemcpyDeviceToHost));
    int status = TPS_OK;
    for (int i = 0; i < n; ++i) {
      CGScalars sc{};
      TPS_CUDA(cudaMemcpy(&sc, B->sys[i]->scalars.p, sizeof(CGScalars), cudaMemcpyDeviceToHost));
      tps_report &r = reports[i];
      std::memset(&r, 0, sizeof(r));
      const double *hi = hist.data() + static_cast<size_t>(i) * TPS_MAX_HISTORY;
      const int nh = std::min(it[i] + 1, TPS_MAX_HISTORY);
      for (int k = 0; k < nh; ++k) r.history[k] = hi[k];
      r.iterations = it[i];
      r.initial_residual = hi[0] * bn[i];
      r.final_residual = std::sqrt(sc.rr) / bn[i];
      r.converged = (sc.breakdown == 0 && r.final_residual <= opts->rel_tol) ? 1 : 0;
      r.time_ms = ms;
      int si = TPS_OK;
      if (sc.breakdown) si = sc.breakdown == 2 ? TPS_ERR_NONFINITE : TPS_ERR_BREAKDOWN;
      else if (!r.converged) si = TPS_ERR_NOT_CONVERGED;
      if (si != TPS_OK && (status == TPS_OK || status == TPS_ERR_NOT_CONVERGED)) status = si;
    }
    for (int i = 0; i < n; ++i)
      if (take_timeout_flag(B->sys[i], s)) {
        reports[i].converged = 0;
        status = TPS_ERR_TIMEOUT;
      }
    (void)act;
    return status;
  });
}

}  // extern "C"
