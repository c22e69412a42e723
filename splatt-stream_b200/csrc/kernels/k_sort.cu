/*
 * k_sort.cu -- exclusive scan and stable LSD radix sort of (key, value) u32
 * pairs.  These order the nonzeros of a CSF (the reference's tt_sort,
 * src/sort.c:761-956, produces the same lexicographic order for distinct
 * coordinates; here a mode-by-mode stable LSD sort reaches it).
 *
 * Radix pass = three launches: per-tile digit histogram, scan of the
 * digit-major count table, stable scatter.  Stability inside a tile: every
 * warp owns a contiguous run of the tile, ranks same-digit lanes with
 * __match_any_sync per 32-item round, and rounds are processed in order.
 */
#include "common.cuh"

namespace sb {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_IPT = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_IPT;

/* exclusive scan of one value per thread across the block */
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t * warp_tot,
    uint32_t * block_total)
{
  int const lane = threadIdx.x & 31;
  int const wid = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for(int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if(lane >= o) { x += y; }
  }
  if(lane == 31) { warp_tot[wid] = x; }
  __syncthreads();
  if(wid == 0) {
    int const nw = blockDim.x >> 5;
    uint32_t t = lane < nw ? warp_tot[lane] : 0;
    uint32_t s = t;
#pragma unroll
    for(int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if(lane >= o) { s += y; }
    }
    if(lane < nw) { warp_tot[lane] = s - t; }
    if(lane == nw - 1) { warp_tot[32] = s; }
  }
  __syncthreads();
  uint32_t const r = x - v + warp_tot[wid];
  if(block_total) { *block_total = warp_tot[32]; }
  __syncthreads();
  return r;
}

__global__ void k_tile_sums(uint32_t const * __restrict__ in, uint64_t n,
    uint32_t * __restrict__ sums)
{
  __shared__ uint32_t wt[33];
  uint64_t const base = (uint64_t) blockIdx.x * SCAN_TILE;
  uint32_t s = 0;
#pragma unroll
  for(int k = 0; k < SCAN_IPT; ++k) {
    uint64_t i = base + (uint64_t) k * SCAN_THREADS + threadIdx.x;
    if(i < n) { s += in[i]; }
  }
  s = warp_sum(s);
  if((threadIdx.x & 31) == 0) { wt[threadIdx.x >> 5] = s; }
  __syncthreads();
  if(threadIdx.x == 0) {
    uint32_t t = 0;
    for(int w = 0; w < SCAN_THREADS / 32; ++w) { t += wt[w]; }
    sums[blockIdx.x] = t;
  }
}

__global__ void k_tile_scan(uint32_t const * __restrict__ in, uint64_t n,
    uint32_t const * __restrict__ offs, uint32_t * __restrict__ out)
{
  __shared__ uint32_t wt[33];
  uint64_t const base = (uint64_t) blockIdx.x * SCAN_TILE + (uint64_t) threadIdx.x * SCAN_IPT;
  uint32_t v[SCAN_IPT];
  uint32_t s = 0;
#pragma unroll
  for(int k = 0; k < SCAN_IPT; ++k) {
    uint64_t i = base + k;
    v[k] = i < n ? in[i] : 0;
    s += v[k];
  }
  uint32_t run = block_excl_scan(s, wt, nullptr) + (offs ? offs[blockIdx.x] : 0);
#pragma unroll
  for(int k = 0; k < SCAN_IPT; ++k) {
    uint64_t i = base + k;
    if(i < n) { out[i] = run; }
    run += v[k];
  }
}

static int excl_scan_rec(uint32_t const * in, uint32_t * out, uint64_t n)
{
  uint64_t const nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  if(nb <= 1) {
    k_tile_scan<<<1, SCAN_THREADS, 0, stream()>>>(in, n, nullptr, out);
    SB_CHECK_LAUNCH();
    return SB_OK;
  }
  uint32_t * sums = nullptr;
  uint32_t * soff = nullptr;
  int rc = talloc(&sums, nb);
  if(rc) { return rc; }
  rc = talloc(&soff, nb);
  if(rc) { tfree(sums); return rc; }
  k_tile_sums<<<(unsigned) nb, SCAN_THREADS, 0, stream()>>>(in, n, sums);
  SB_CHECK_LAUNCH();
  rc = excl_scan_rec(sums, soff, nb);
  if(rc == SB_OK) {
    k_tile_scan<<<(unsigned) nb, SCAN_THREADS, 0, stream()>>>(in, n, soff, out);
    if(cudaGetLastError() != cudaSuccess) { rc = SB_EDEVICE; }
  }
  tfree(sums);
  tfree(soff);
  return rc;
}

/* ---------------------------- radix sort -------------------------------- */
constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ROUNDS = 16;                       /* 32-item rounds per warp */
constexpr int RS_TILE = RS_THREADS * RS_ROUNDS;     /* 4096 items per block */

__global__ void __launch_bounds__(RS_THREADS)
k_radix_hist(uint32_t const * __restrict__ keys, uint64_t n, int shift,
    uint32_t * __restrict__ counts, uint32_t nblocks)
{
  __shared__ uint32_t hist[256];
  hist[threadIdx.x] = 0;
  __syncthreads();
  uint64_t const base = (uint64_t) blockIdx.x * RS_TILE;
#pragma unroll 4
  for(int r = 0; r < RS_ROUNDS; ++r) {
    uint64_t i = base + (uint64_t) r * RS_THREADS + threadIdx.x;
    if(i < n) { atomicAdd(&hist[(keys[i] >> shift) & 0xffu], 1u); }
  }
  __syncthreads();
  counts[(uint64_t) threadIdx.x * nblocks + blockIdx.x] = hist[threadIdx.x];
}

__global__ void __launch_bounds__(RS_THREADS)
k_radix_scatter(uint32_t const * __restrict__ kin, uint32_t const * __restrict__ vin,
    uint32_t * __restrict__ kout, uint32_t * __restrict__ vout, uint64_t n,
    int shift, uint32_t const * __restrict__ offs, uint32_t nblocks)
{
  __shared__ uint32_t wcnt[RS_WARPS][256];
  int const lane = threadIdx.x & 31;
  int const wid = threadIdx.x >> 5;
  for(int d = threadIdx.x; d < RS_WARPS * 256; d += RS_THREADS) {
    (&wcnt[0][0])[d] = 0;
  }
  __syncthreads();

  uint64_t const wbase = (uint64_t) blockIdx.x * RS_TILE + (uint64_t) wid * (32 * RS_ROUNDS);
  uint32_t key[RS_ROUNDS], val[RS_ROUNDS], dig[RS_ROUNDS];
#pragma unroll
  for(int r = 0; r < RS_ROUNDS; ++r) {
    uint64_t i = wbase + (uint64_t) r * 32 + lane;
    bool const ok = i < n;
    key[r] = ok ? kin[i] : 0u;
    val[r] = ok ? vin[i] : 0u;
    dig[r] = ok ? ((key[r] >> shift) & 0xffu) : 256u;
  }
  /* phase A: per-warp digit counts */
#pragma unroll
  for(int r = 0; r < RS_ROUNDS; ++r) {
    unsigned const peers = __match_any_sync(0xffffffffu, dig[r]);
    if(dig[r] < 256u && lane == __ffs(peers) - 1) {
      wcnt[wid][dig[r]] += __popc(peers);
    }
    __syncwarp();
  }
  __syncthreads();
  /* phase B: per digit, warp-major prefix from the block's global offset */
  {
    int const d = threadIdx.x;
    uint32_t run = offs[(uint64_t) d * nblocks + blockIdx.x];
#pragma unroll
    for(int w = 0; w < RS_WARPS; ++w) {
      uint32_t c = wcnt[w][d];
      wcnt[w][d] = run;
      run += c;
    }
  }
  __syncthreads();
  /* phase C: stable scatter, rounds in order */
  unsigned const lt = lanemask_lt();
#pragma unroll
  for(int r = 0; r < RS_ROUNDS; ++r) {
    unsigned const peers = __match_any_sync(0xffffffffu, dig[r]);
    if(dig[r] < 256u) {
      uint32_t const pos = wcnt[wid][dig[r]] + __popc(peers & lt);
      kout[pos] = key[r];
      vout[pos] = val[r];
    }
    __syncwarp();
    if(dig[r] < 256u && lane == __ffs(peers) - 1) {
      wcnt[wid][dig[r]] += __popc(peers);
    }
    __syncwarp();
  }
}

} /* namespace sb */

using namespace sb;

extern "C" {

int sb_exclusive_scan_u32(uint32_t const * in, uint32_t * out, uint64_t n,
    uint64_t * total)
{
  if(n == 0) {
    if(total) { *total = 0; }
    return SB_OK;
  }
  int rc = excl_scan_rec(in, out, n);
  if(rc) { return rc; }
  if(total) {
    uint32_t last_in = 0, last_out = 0;
    SB_TRY(cudaMemcpyAsync(&last_in, in + n - 1, 4, cudaMemcpyDeviceToHost, stream()));
    SB_TRY(cudaMemcpyAsync(&last_out, out + n - 1, 4, cudaMemcpyDeviceToHost, stream()));
    SB_TRY(cudaStreamSynchronize(stream()));
    *total = (uint64_t) last_in + last_out;
  }
  return SB_OK;
}

int sb_radix_sort_pairs(uint32_t * keys, uint32_t * vals, uint32_t * keys_alt,
    uint32_t * vals_alt, uint64_t n, int bits, int * result_in_alt)
{
  *result_in_alt = 0;
  if(n <= 1 || bits <= 0) { return SB_OK; }
  if(n >= 0xffffffffull) { return SB_EINPUT; }
  uint32_t const nb = (uint32_t) ((n + RS_TILE - 1) / RS_TILE);
  uint64_t const ncount = 256ull * nb;
  uint32_t * counts = nullptr, * offs = nullptr;
  int rc = talloc(&counts, ncount);
  if(rc) { return rc; }
  rc = talloc(&offs, ncount);
  if(rc) { tfree(counts); return rc; }
  uint32_t * ki = keys, * vi = vals, * ko = keys_alt, * vo = vals_alt;
  int flip = 0;
  for(int shift = 0; shift < bits; shift += 8) {
    k_radix_hist<<<nb, RS_THREADS, 0, stream()>>>(ki, n, shift, counts, nb);
    if(cudaGetLastError() != cudaSuccess) { rc = SB_EDEVICE; break; }
    rc = excl_scan_rec(counts, offs, ncount);
    if(rc) { break; }
    k_radix_scatter<<<nb, RS_THREADS, 0, stream()>>>(ki, vi, ko, vo, n, shift, offs, nb);
    if(cudaGetLastError() != cudaSuccess) { rc = SB_EDEVICE; break; }
    uint32_t * t;
    t = ki; ki = ko; ko = t;
    t = vi; vi = vo; vo = t;
    flip ^= 1;
  }
  tfree(counts);
  tfree(offs);
  *result_in_alt = flip;
  return rc;
}

} /* extern "C" */
