/*
 * common.cuh -- shared helpers for the sm_100a kernels.
 */
#ifndef SPLATT_B200_COMMON_CUH
#define SPLATT_B200_COMMON_CUH

#include <cuda_runtime.h>
#include <stdint.h>
#include "kapi.h"

namespace sb {

/* The library's current stream (set by sb_set_stream; default: a stream
 * created by sb_init). */
cudaStream_t stream();

/* Record a CUDA error and map it to an SB_* code. */
int fail(cudaError_t e);

#define SB_TRY(expr)                         \
  do {                                       \
    cudaError_t sb_e_ = (expr);              \
    if(sb_e_ != cudaSuccess) {               \
      return ::sb::fail(sb_e_);              \
    }                                        \
  } while(0)

#define SB_CHECK_LAUNCH() SB_TRY(cudaGetLastError())

/* stream-ordered temporary allocation */
template <typename T>
inline int talloc(T ** p, size_t n)
{
  if(n == 0) { n = 1; }
  cudaError_t e = cudaMallocAsync((void **) p, n * sizeof(T), stream());
  if(e != cudaSuccess) { return fail(e); }
  return SB_OK;
}

template <typename T>
inline void tfree(T * p)
{
  if(p) { cudaFreeAsync(p, stream()); }
}

inline unsigned blocks_for(uint64_t n, unsigned threads)
{
  uint64_t b = (n + threads - 1) / threads;
  return (unsigned) (b == 0 ? 1 : b);
}

__device__ __forceinline__ unsigned lanemask_lt()
{
  unsigned m;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__host__ __device__ __forceinline__ uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ uint32_t umin32(uint32_t a, uint32_t b) { return a < b ? a : b; }

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
  for(int o = 16; o > 0; o >>= 1) {
    v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  return v;
}

/* first index k in [0, n) with a[k] > x (a sorted ascending); n if none */
__device__ __forceinline__ uint32_t upper_bound_u32(uint32_t const * a,
    uint32_t n, uint32_t x)
{
  uint32_t lo = 0, hi = n;
  while(lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if(__ldg(a + mid) <= x) { lo = mid + 1; } else { hi = mid; }
  }
  return lo;
}

} /* namespace sb */

#endif
