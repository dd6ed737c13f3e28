// Kernel launches with programmatic dependent launch (sm_90 and later).
//
// Every kernel of this library starts with griddep_wait(), before its first
// global-memory access, and every launch carries the programmatic stream
// serialization attribute.  A kernel may then be launched, and its CTAs
// scheduled, while the previous kernel in the stream is still finishing;
// griddep_wait() returns once that grid has completed and its memory
// operations are visible.  Inside the CUDA graphs of the solvers the launch
// latency of each of the many small dependent kernels of a V-cycle (the
// coarse levels are latency-bound) overlaps its predecessor's tail.  Launched
// without the attribute, griddep_wait() returns at once.
#pragma once

#include <cuda_runtime.h>

#include <utility>

#ifndef TPS_PDL
#define TPS_PDL 1  // 0: plain stream-ordered launches (same kernels)
#endif
// 1: each CTA also allows the next kernel's launch right after its wait.
// Measured slower (CG 64^3 FP64 24.57 vs 23.16 ms, 16^3 FP32 1.78 vs 1.65
// ms): the waiting dependent CTAs take SM resources from the running grid.
#ifndef TPS_PDL_EARLY
#define TPS_PDL_EARLY 0
#endif

namespace tps {

__device__ __forceinline__ void griddep_wait()
{
#if defined(__CUDA_ARCH__)
  asm volatile("griddepcontrol.wait;" ::: "memory");
#if TPS_PDL_EARLY
  // the dependent grid may launch once every CTA of this grid has passed
  // here; its CTAs then wait in their own griddep_wait() for this grid's end
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
#endif
}

// launch errors are recorded like those of <<< >>> launches and are read by
// the callers' cudaGetLastError()
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args &&...args)
{
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = TPS_PDL;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

}  // namespace tps

#define TPS_LAUNCH(kern, grid, block, smem, stream, ...) \
  ((void)::tps::launch_pdl(kern, grid, block, smem, stream, ##__VA_ARGS__))
