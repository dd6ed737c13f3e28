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
  void *scratch = nullptr;        // device address of g_noalloc_scratch on this device
  unsigned degrees_uploaded = 0;  // bit k: tables of degree k are in constant memory
};

std::mutex g_mutex;
DeviceState g_state[kMaxDevices];

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
    // per-device set-up on the first call (the current device is `dev`)
    std::lock_guard<std::mutex> lock(g_mutex);
    DeviceState &st = g_state[dev];
    if (!st.scratch) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess) return fail(TPS_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      st.scratch = p;
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
