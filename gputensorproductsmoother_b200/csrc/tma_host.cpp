// Host-side TMA descriptor encoding (cuTensorMapEncodeTiled obtained through
// cudaGetDriverEntryPoint, so the library links against the runtime only).
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "kernel_table.h"

namespace tps {
namespace {

using EncodeFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                              const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                              const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                              CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encode_fn(cudaError_t &err)
{
  static EncodeFn fn = nullptr;
  static cudaError_t status = cudaSuccess;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    status = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
    if (status == cudaSuccess && q != cudaDriverEntryPointSuccess) status = cudaErrorNotSupported;
    fn = reinterpret_cast<EncodeFn>(p);
  });
  err = status;
  return fn;
}

}  // namespace

cudaError_t encode_tiled(void *map_out, bool f64, void *base, int rank, const uint64_t *dims,
                         const uint64_t *strides_bytes, const uint32_t *box)
{
  if (rank < 3 || rank > 5) return cudaErrorInvalidValue;
  cudaError_t e;
  EncodeFn fn = encode_fn(e);
  if (!fn) return e == cudaSuccess ? cudaErrorNotSupported : e;
  cuuint64_t gdim[5], gstr[4];
  cuuint32_t bdim[5], estr[5];
  for (int i = 0; i < rank; ++i) {
    gdim[i] = dims[i];
    bdim[i] = box[i];
    estr[i] = 1;
    if (i + 1 < rank) gstr[i] = strides_bytes[i];
  }
  CUresult r = fn(reinterpret_cast<CUtensorMap *>(map_out),
                  f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                  static_cast<cuuint32_t>(rank), base, gdim, gstr, bdim, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

}  // namespace tps
