/*
 * k_ingest.cu -- the streaming parser's preparation of a tensor on the device.
 *
 * Replaces ParserSimple's constructor and next_batch bookkeeping
 * (src/cpd/stream/ParserSimple.cc:13-79, 89-149), which splatt_cpd_stream ran
 * on the host (a comparison sort of every nonzero, then a serial relabel):
 *   1. order the nonzeros by (stream mode, then the following modes
 *      cyclically): LSD radix passes over the mode keys, least significant
 *      first, carrying a permutation (the same passes as the CSF build);
 *   2. relabel every other mode by first appearance in that order: the first
 *      position of each index (atomicMin), a mark on the positions that are
 *      first occurrences, an exclusive scan of the marks = the new label;
 *   3. the slice boundaries (lower bounds of each time index in the sorted
 *      time column) and, per slice, the number of labels seen up to its end,
 *      which is the dims[m] = max(max index + 1, previous dims) that
 *      next_batch reports (labels appear in increasing order).
 */
#include "common.cuh"

namespace sb {
namespace {

__global__ void k_ing_iota(uint32_t * p, uint64_t n)
{
  uint64_t const i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(i < n) { p[i] = (uint32_t) i; }
}

__global__ void k_ing_gather_u32(uint32_t const * __restrict__ src,
    uint32_t const * __restrict__ perm, uint32_t * __restrict__ dst, uint64_t n)
{
  uint64_t const i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(i < n) { dst[i] = src[perm[i]]; }
}

template <typename T>
__global__ void k_ing_gather_val(T const * __restrict__ src, uint32_t const * __restrict__ perm,
    T * __restrict__ dst, uint64_t n)
{
  uint64_t const i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(i < n) { dst[i] = src[perm[i]]; }
}

__global__ void k_ing_fill(uint32_t * p, uint64_t n, uint32_t v)
{
  uint64_t const i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(i < n) { p[i] = v; }
}

/* first position of every index value */
__global__ void k_ing_first(uint32_t const * __restrict__ ind, uint64_t n,
    uint32_t * __restrict__ first)
{
  uint64_t const i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(i < n) { atomicMin(first + ind[i], (uint32_t) i); }
}

/* 1 where a position is its index's first occurrence */
__global__ void k_ing_mark(uint32_t const * __restrict__ ind, uint64_t n,
    uint32_t const * __restrict__ first, uint32_t * __restrict__ mark)
{
  uint64_t const i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(i < n) { mark[i] = first[ind[i]] == (uint32_t) i ? 1u : 0u; }
}

/* new label = rank of the index's first occurrence; iperm[label] = index */
__global__ void k_ing_relabel(uint32_t * __restrict__ ind, uint64_t n,
    uint32_t const * __restrict__ first, uint32_t const * __restrict__ rank,
    uint32_t const * __restrict__ mark, uint32_t * __restrict__ iperm)
{
  uint64_t const i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n) { return; }
  uint32_t const v = ind[i];
  if(mark[i]) { iperm[rank[i]] = v; }
  ind[i] = rank[first[v]];
}

/* offs[t] = first position whose time index is >= t, t = 0..T */
__global__ void k_ing_bounds(uint32_t const * __restrict__ time, uint64_t n, uint64_t T,
    uint64_t * __restrict__ offs)
{
  uint64_t const t = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(t > T) { return; }
  uint64_t lo = 0, hi = n;
  while(lo < hi) {
    uint64_t const mid = (lo + hi) >> 1;
    if((uint64_t) time[mid] < t) { lo = mid + 1; } else { hi = mid; }
  }
  offs[t] = lo;
}

/* labels seen up to the end of slice t: rank + mark at its last position */
__global__ void k_ing_seen(uint64_t const * __restrict__ offs, uint64_t T,
    uint32_t const * __restrict__ rank, uint32_t const * __restrict__ mark,
    uint64_t * __restrict__ seen)
{
  uint64_t const t = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(t >= T) { return; }
  uint64_t const e = offs[t + 1];
  seen[t] = e ? (uint64_t) rank[e - 1] + mark[e - 1] : 0;
}

int ing_bits(uint64_t x)
{
  int b = 0;
  while(b < 64 && (1ull << b) < x) { ++b; }
  return b;
}

} /* namespace */
} /* namespace sb */

using namespace sb;

extern "C" {

int sb_stream_prepare(uint32_t nmodes, uint64_t nnz, uint64_t const * dims,
    uint32_t * const * inds, void const * vals, int vt, uint32_t sm,
    uint32_t * const * out_inds, void * out_vals, uint32_t * const * iperm,
    uint64_t * nlabels, uint64_t * offs, uint64_t * seen)
{
  if(nmodes < 2 || nmodes > SB_MAX_NMODES || sm >= nmodes || nnz == 0 ||
      nnz >= 0xffffffffull) {
    return SB_EINPUT;
  }
  for(uint32_t m = 0; m < nmodes; ++m) {
    if(dims[m] == 0 || dims[m] >= 0xffffffffull) { return SB_EINPUT; }
  }
  cudaStream_t s = stream();
  unsigned const nb = blocks_for(nnz, 256);
  uint64_t const T = dims[sm];
  uint32_t * perm = nullptr, * perm2 = nullptr, * keys = nullptr, * keys2 = nullptr;
  uint32_t * first = nullptr, * mark = nullptr, * rank = nullptr;
  uint64_t * doffs = nullptr, * dseen = nullptr;
  uint64_t maxdim = 1;
  for(uint32_t m = 0; m < nmodes; ++m) { if(dims[m] > maxdim) { maxdim = dims[m]; } }
  int rc = SB_OK;
#define SB_STEP(x) do { rc = (x); if(rc) { goto done; } } while(0)
  SB_STEP(talloc(&perm, nnz));
  SB_STEP(talloc(&perm2, nnz));
  SB_STEP(talloc(&keys, nnz));
  SB_STEP(talloc(&keys2, nnz));
  k_ing_iota<<<nb, 256, 0, s>>>(perm, nnz);
  /* 1. (sm, sm+1, ...) order: least significant key first */
  for(int l = (int) nmodes - 1; l >= 0; --l) {
    uint32_t const m = (sm + (uint32_t) l) % nmodes;
    int const bits = ing_bits(dims[m]);
    if(bits == 0) { continue; }
    k_ing_gather_u32<<<nb, 256, 0, s>>>(inds[m], perm, keys, nnz);
    int alt = 0;
    SB_STEP(sb_radix_sort_pairs(keys, perm, keys2, perm2, nnz, bits, &alt));
    if(alt) {
      uint32_t * t = perm; perm = perm2; perm2 = t;
      t = keys; keys = keys2; keys2 = t;
    }
  }
  for(uint32_t m = 0; m < nmodes; ++m) {
    k_ing_gather_u32<<<nb, 256, 0, s>>>(inds[m], perm, out_inds[m], nnz);
  }
  if(vt == SB_F64) {
    k_ing_gather_val<double><<<nb, 256, 0, s>>>((double const *) vals, perm, (double *) out_vals, nnz);
  } else {
    k_ing_gather_val<float><<<nb, 256, 0, s>>>((float const *) vals, perm, (float *) out_vals, nnz);
  }
  /* 3a. slice bounds from the sorted time column */
  SB_STEP(talloc(&doffs, T + 1));
  SB_STEP(talloc(&dseen, T ? T : 1));
  k_ing_bounds<<<blocks_for(T + 1, 256), 256, 0, s>>>(out_inds[sm], nnz, T, doffs);
  /* 2. first-appearance labels of the other modes */
  SB_STEP(talloc(&first, maxdim));
  SB_STEP(talloc(&mark, nnz));
  SB_STEP(talloc(&rank, nnz));
  for(uint32_t m = 0; m < nmodes; ++m) {
    nlabels[m] = 0;
    if(m == sm) { continue; }
    k_ing_fill<<<blocks_for(dims[m], 256), 256, 0, s>>>(first, dims[m], 0xffffffffu);
    k_ing_first<<<nb, 256, 0, s>>>(out_inds[m], nnz, first);
    k_ing_mark<<<nb, 256, 0, s>>>(out_inds[m], nnz, first, mark);
    uint64_t total = 0;
    SB_STEP(sb_exclusive_scan_u32(mark, rank, nnz, &total));
    nlabels[m] = total;
    k_ing_relabel<<<nb, 256, 0, s>>>(out_inds[m], nnz, first, rank, mark, iperm[m]);
    /* 3b. labels seen up to each slice end (pageable host copy: the call
     * returns once it has landed, so dseen can be reused for the next mode) */
    if(T) {
      k_ing_seen<<<blocks_for(T, 256), 256, 0, s>>>(doffs, T, rank, mark, dseen);
      SB_STEP(cudaMemcpyAsync(seen + (size_t) m * T, dseen, T * sizeof(uint64_t),
                              cudaMemcpyDeviceToHost, s) == cudaSuccess ? SB_OK : SB_EDEVICE);
      SB_STEP(cudaStreamSynchronize(s) == cudaSuccess ? SB_OK : SB_EDEVICE);
    }
  }
  SB_STEP(cudaMemcpyAsync(offs, doffs, (T + 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost, s) ==
          cudaSuccess ? SB_OK : SB_EDEVICE);
  SB_STEP(cudaGetLastError() == cudaSuccess ? SB_OK : SB_EDEVICE);
  SB_STEP(cudaStreamSynchronize(s) == cudaSuccess ? SB_OK : SB_EDEVICE);
done:
#undef SB_STEP
  tfree(perm); tfree(perm2); tfree(keys); tfree(keys2);
  tfree(first); tfree(mark); tfree(rank); tfree(doffs); tfree(dseen);
  return rc;
}

} /* extern "C" */
