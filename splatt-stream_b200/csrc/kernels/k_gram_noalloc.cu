/*
 * k_gram_noalloc.cu -- the Gram matrix G = A^T A without any device
 * allocation: splatt_b200_gram_noalloc.
 *
 * Why it exists.  The regular Gram entry point (sb_gram) asks the CUDA
 * stream-ordered allocator for a buffer of per-block partial sums on every
 * call.  Some callers cannot do that:
 *   - a serving process that has already divided all of its device memory
 *     between resident stream state and its own pools, so one more
 *     allocation either fails or eats into another stream's budget;
 *   - a plug-in loaded into a host application that owns the allocator
 *     policy and forbids libraries from calling cudaMalloc / cudaFree
 *     behind its back (cudaFree can also stall the whole device, which a
 *     latency-bound caller cannot accept).
 * This variant keeps the partial sums in one file-scope device array
 * instead, so a call allocates nothing: the caller passes A and G, and the
 * scratch is the fixed array below.
 *
 * Limits and sharing.  The scratch holds SB_NOALLOC_MAX_BLOCKS partial
 * R x R blocks for R <= SB_NOALLOC_MAX_R: 64 x 64 x 64 doubles = 2 MiB, held
 * by every GPU that loads the library until the process exits.  Ranks above
 * SB_NOALLOC_MAX_R are rejected (SPLATT_ERROR_BADINPUT plus a message on
 * stderr); the number of rows is unlimited (blocks loop over row tiles).
 * Every call on a device shares the same array and leaves its contents
 * behind: two calls whose kernels overlap on the GPU (different streams, or
 * host threads racing) corrupt each other's partial sums, so callers must
 * order their calls on one stream or otherwise serialise them.  Nothing in
 * the scratch has to start at zero: each call writes every partial it later
 * reads; the output G is cleared by the call itself.
 *
 * Set-up.  Host code cannot use the array's name as a device address (in
 * host code it is only a stand-in symbol).  The first call on each device
 * looks the device address up with cudaGetSymbolAddress, with that device
 * current, and caches it; that first call should therefore be made before
 * any stream capture is started.  The cached address belongs to the device's
 * primary context: after cudaDeviceReset (or anything else that destroys
 * and recreates that context) it no longer points at the array, so a process
 * that resets a device must not call this entry point on it again.
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../../../include/splatt_b200.h"

#define SB_NOALLOC_MAX_R 64
#define SB_NOALLOC_MAX_BLOCKS 64
#define SB_NOALLOC_ROWS 64
#define SB_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) double
    g_gram_scratch[SB_NOALLOC_MAX_BLOCKS * SB_NOALLOC_MAX_R * SB_NOALLOC_MAX_R];

/* device address of g_gram_scratch, per device (0 until looked up) */
static double * g_scratch_addr[SB_NOALLOC_MAX_DEVICES];

/* part[b][i*R + j] (j >= i) = sum over block b's row tiles of A[r][i] A[r][j] */
template <typename T>
__global__ void __launch_bounds__(256)
k_gram_noalloc_partial(T const * __restrict__ A, uint64_t I, uint32_t R, uint32_t ld,
    double * __restrict__ part)
{
  __shared__ double tile[SB_NOALLOC_ROWS * SB_NOALLOC_MAX_R];
  uint32_t const npairs = R * (R + 1) / 2;
  double acc[9];
  uint32_t pi[9], pj[9];
  int np = 0;
  /* 64 x 65 / 2 = 2080 pairs over 256 threads: at most 9 per thread */
  for(uint32_t p = threadIdx.x; p < npairs && np < 9; p += blockDim.x, ++np) {
    uint32_t i = 0, rem = p;
    while(rem >= R - i) { rem -= R - i; ++i; }
    pi[np] = i;
    pj[np] = i + rem;
    acc[np] = 0.;
  }
  for(uint64_t r0 = (uint64_t) blockIdx.x * SB_NOALLOC_ROWS; r0 < I;
      r0 += (uint64_t) gridDim.x * SB_NOALLOC_ROWS) {
    uint32_t const nr = (uint32_t) ((I - r0) < SB_NOALLOC_ROWS ? (I - r0) : SB_NOALLOC_ROWS);
    __syncthreads();
    for(uint32_t e = threadIdx.x; e < nr * R; e += blockDim.x) {
      uint32_t const rr = e / R, cc = e % R;
      tile[rr * R + cc] = (double) A[(r0 + rr) * ld + cc];
    }
    __syncthreads();
    for(int q = 0; q < np; ++q) {
      double s = acc[q];
      for(uint32_t rr = 0; rr < nr; ++rr) { s = fma(tile[rr * R + pi[q]], tile[rr * R + pj[q]], s); }
      acc[q] = s;
    }
  }
  double * P = part + (size_t) blockIdx.x * R * R;
  for(int q = 0; q < np; ++q) { P[pi[q] * R + pj[q]] = acc[q]; }
}

/* G[i*R + j] (j >= i) = sum over the nb partial blocks, in block order */
__global__ void k_gram_noalloc_reduce(double const * __restrict__ part, uint32_t nb,
    uint32_t R, double * __restrict__ G)
{
  uint32_t const e = blockIdx.x * blockDim.x + threadIdx.x;
  if(e >= R * R) { return; }
  if(e % R < e / R) { return; }
  double s = 0.;
  for(uint32_t b = 0; b < nb; ++b) { s += part[(size_t) b * R * R + e]; }
  G[e] = s;
}

extern "C" splatt_error_type splatt_b200_gram_noalloc(void const * A, int val_type,
    uint64_t nrows, uint32_t rank, uint32_t ld, double * G, void * cuda_stream)
{
  if(A == NULL || G == NULL || rank == 0 || ld < rank || (val_type != 0 && val_type != 1)) {
    return SPLATT_ERROR_BADINPUT;
  }
  if(rank > SB_NOALLOC_MAX_R) {
    fprintf(stderr, "splatt_b200_gram_noalloc: rank %u exceeds the supported maximum %d\n",
        rank, SB_NOALLOC_MAX_R);
    return SPLATT_ERROR_BADINPUT;
  }
  cudaStream_t const st = (cudaStream_t) cuda_stream;
  int dev = 0;
  if(cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= SB_NOALLOC_MAX_DEVICES) {
    cudaGetLastError();
    return SPLATT_ERROR_DEVICE;
  }
  if(g_scratch_addr[dev] == NULL) {
    void * p = NULL;
    cudaError_t const e = cudaGetSymbolAddress(&p, g_gram_scratch);
    if(e != cudaSuccess || p == NULL) {
      cudaGetLastError();
      return SPLATT_ERROR_DEVICE;
    }
    g_scratch_addr[dev] = (double *) p;
  }
  double * const part = g_scratch_addr[dev];

  if(cudaMemsetAsync(G, 0, (size_t) rank * rank * sizeof(double), st) != cudaSuccess) {
    cudaGetLastError();
    return SPLATT_ERROR_DEVICE;
  }
  if(nrows == 0) { return SPLATT_SUCCESS; }
  uint64_t const tiles = (nrows + SB_NOALLOC_ROWS - 1) / SB_NOALLOC_ROWS;
  unsigned const nb = (unsigned) (tiles < SB_NOALLOC_MAX_BLOCKS ? tiles : SB_NOALLOC_MAX_BLOCKS);
  if(val_type == 0) {
    k_gram_noalloc_partial<double><<<nb, 256, 0, st>>>((double const *) A, nrows, rank, ld, part);
  } else {
    k_gram_noalloc_partial<float><<<nb, 256, 0, st>>>((float const *) A, nrows, rank, ld, part);
  }
  k_gram_noalloc_reduce<<<(rank * rank + 255) / 256, 256, 0, st>>>(part, nb, rank, G);
  if(cudaGetLastError() != cudaSuccess) { return SPLATT_ERROR_DEVICE; }
  return SPLATT_SUCCESS;
}
