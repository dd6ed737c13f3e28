// Division by a run-time invariant as a multiply and shift.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace tps {

// The round-up method of Granlund & Montgomery ("Division by invariant
// integers using multiplication", PLDI 1994, Thm. 4.2 with N = 31): with
// l = ceil(log2 d), s = 31 + l and m = ceil(2^s / d) < 2^32,
// floor(n m / 2^s) = floor(n / d) for every 0 <= n < 2^31 and d >= 1.
inline void magic_div(uint32_t d, uint32_t &m, uint32_t &s)
{
  uint32_t l = 0;
  while ((uint64_t(1) << l) < d) ++l;
  s = 31 + l;
  m = static_cast<uint32_t>(((uint64_t(1) << s) + d - 1) / d);
}

__host__ __device__ __forceinline__ int fast_div(int n, uint32_t m, uint32_t s)
{
  return static_cast<int>((static_cast<uint64_t>(static_cast<uint32_t>(n)) * m) >> s);
}

}  // namespace tps
