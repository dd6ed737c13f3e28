// Restriction entry point that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc: hosts whose framework
// owns all device memory (a caching allocator or a fixed arena reserved at
// start-up) and forbids allocations it does not manage.  tps_restrict_add
// needs a handle whose work vectors (including the 3D transfer intermediate)
// are allocated on first use; this variant needs no handle and keeps the
// intermediate in the file-scope array below instead, so it only touches the
// caller's input and output buffers plus that fixed array.
//
// The array is kTpsNoallocScratchBytes (16 MiB) and every GPU that loads the
// library holds it until the process exits.  All calls share it: calls whose
// executions overlap on the GPU (different streams, or different host
// threads) race on it and must be serialised by the caller.  It needs no
// clearing: every entry the z pass reads is written by the xy pass of the same
// call first.
//
// Set-up: every call looks up the array's device address in the current
// context (cudaGetSymbolAddress, a host-side lookup).  The 1D tables of a
// degree are uploaded to constant memory on the first call on a device and
// again whenever the device's CUDA context has changed since (cudaDeviceReset
// unloads the module, so the uploaded tables are gone); the context is
// identified by cuCtxGetId.  A first call on a device therefore copies tables
// to the device: make it before any stream capture.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "../../include/tps.h"
#include "fe_data.h"
#include "kernel_table.h"

namespace tps {

// thread-local message reported by tps_last_error(NULL) (defined with the ABI)
void set_handle_free_error(const std::string &msg);

constexpr size_t kTpsNoallocScratchBytes = size_t(16) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kTpsNoallocScratchBytes];

namespace {

constexpr int kMaxDevices = 64;

struct DeviceState {
  unsigned long long ctx_id = 0;  // context the entries below belong to
  bool ready = false;             // set-up done for ctx_id
  void *scratch = nullptr;        // device address of g_noalloc_scratch in that context
  unsigned degrees_uploaded = 0;  // bit k: tables of degree k are in its constant memory
};

std::mutex g_mutex;
DeviceState g_state[kMaxDevices];

using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);

// unique id of the calling thread's current context (driver entry points
// obtained through the runtime, so the library links the runtime only)
cudaError_t current_context_id(unsigned long long &id)
{
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static cudaError_t status = cudaSuccess;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr, *q = nullptr;
    cudaDriverEntryPointQueryResult r1, r2;
    status = cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &r1);
    if (status == cudaSuccess) status = cudaGetDriverEntryPoint("cuCtxGetId", &q, cudaEnableDefault, &r2);
    if (status == cudaSuccess && (r1 != cudaDriverEntryPointSuccess || r2 != cudaDriverEntryPointSuccess))
      status = cudaErrorNotSupported;
    get_current = reinterpret_cast<CtxGetCurrentFn>(p);
    get_id = reinterpret_cast<CtxGetIdFn>(q);
  });
  if (status != cudaSuccess) return status;
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return cudaErrorDeviceUninitialized;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return cudaErrorDeviceUninitialized;
  return cudaSuccess;
}

int fail(int status, const std::string &msg)
{
  set_handle_free_error(msg);
  return status;
}

}  // namespace
}  // namespace tps

using namespace tps;

extern "C" int tps_restrict_add_noalloc(int dim, int degree, int n_coarse_cells, int dtype,
                                        void *coarse, const void *fine, void *stream)
{
  set_handle_free_error("");
  if (dim != 2 && dim != 3) return fail(TPS_ERR_INVALID, "dim must be 2 or 3");
  if (degree < 1 || degree > kMaxDegree) return fail(TPS_ERR_UNSUPPORTED, "degree must be in 1..7");
  if (n_coarse_cells < 1) return fail(TPS_ERR_INVALID, "n_coarse_cells must be >= 1");
  if (dtype != TPS_F64 && dtype != TPS_F32) return fail(TPS_ERR_INVALID, "bad dtype");
  if (!coarse || !fine) return fail(TPS_ERR_INVALID, "null vector");
  const size_t es = dtype == TPS_F64 ? 8 : 4;
  const int64_t N1c = int64_t(n_coarse_cells) * degree + 1;
  const int64_t N1f = 2 * int64_t(n_coarse_cells) * degree + 1;
  // the launch geometry: DoFs per direction as int, coarse-cell tiles of the
  // xy pass as grid x/y (at most 65535 in y)
  if (N1f > INT32_MAX) return fail(TPS_ERR_INVALID, "n_coarse_cells too large: the fine level exceeds 2^31-1 DoFs per direction");
  const int64_t tile_cells = degree <= 4 ? 8 : 4;
  if ((int64_t(n_coarse_cells) + tile_cells - 1) / tile_cells > 65535)
    return fail(TPS_ERR_INVALID, "n_coarse_cells too large for the restriction grid (at most " +
                                     std::to_string(65535 * tile_cells) + " coarse cells per direction)");
  const size_t need = dim == 3 ? es * size_t(N1f) * size_t(N1c) * size_t(N1c) : 0;
  if (need > kTpsNoallocScratchBytes)
    return fail(TPS_ERR_INVALID, "problem needs " + std::to_string(need) +
                                     " scratch bytes; the fixed scratch array holds " +
                                     std::to_string(kTpsNoallocScratchBytes));
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(TPS_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(TPS_ERR_CUDA, "device ordinal out of range");
  const KernelTable *kt = kernel_table(degree);
  void *scratch = nullptr;
  {
    // per-device set-up on the first call in the device's current context
    // (the current device is `dev`)
    std::lock_guard<std::mutex> lock(g_mutex);
    DeviceState &st = g_state[dev];
    // the symbol lookup also makes the device's primary context current
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return fail(TPS_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    unsigned long long ctx = 0;
    e = current_context_id(ctx);
    if (e != cudaSuccess) return fail(TPS_ERR_CUDA, std::string("context id: ") + cudaGetErrorString(e));
    if (!st.ready || st.ctx_id != ctx || st.scratch != p) {
      st = DeviceState{};
      st.scratch = p;
      st.ctx_id = ctx;
      st.ready = true;
    }
    if (!(st.degrees_uploaded & (1u << degree))) {
      static DegreeData tables[kMaxDegree + 1];
      if (tables[degree].k != degree) tables[degree] = make_degree_data(degree);
      e = kt->upload(tables[degree]);
      if (e != cudaSuccess) return fail(TPS_ERR_CUDA, std::string("table upload: ") + cudaGetErrorString(e));
      st.degrees_uploaded |= 1u << degree;
    }
    scratch = st.scratch;
  }
  LevelGeomH gc;
  gc.n = n_coarse_cells;
  gc.N1 = static_cast<int>(N1c);
  gc.N = dim == 3 ? N1c * N1c * N1c : N1c * N1c;
  gc.h = 1.0 / n_coarse_cells;
  const VecLayout lc{static_cast<int>(N1c), N1c, N1c * N1c};
  const VecLayout lf{static_cast<int>(N1f), N1f, N1f * N1f};
  e = kt->restrict_[dim - 2][dtype == TPS_F64 ? 0 : 1](gc, lc, lf, coarse, fine, scratch, 1,
                                                       static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return fail(TPS_ERR_CUDA, cudaGetErrorString(e));
  return TPS_OK;
}
