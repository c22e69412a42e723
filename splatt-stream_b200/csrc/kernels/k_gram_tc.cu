/*
 * k_gram_tc.cu -- G = A^T A of an FP32 factor (rows x R, R <= 64, row-major,
 * leading dimension ld) on the 5th-generation tensor cores (tcgen05,
 * kind::tf32), with split products for FP32 accuracy.
 *
 * Replaces mat_aTa (src/matrix.c:171-205, a dsyrk over the factor) for the
 * FP32 precision mode: "Grams via split TF32 products".
 *
 * Split: every element x = hi + lo with hi = tf32(x), lo = tf32(x - hi)
 * (round to nearest).  One shared-memory operand tile per chunk of 32 rows
 * holds the two halves as MMA rows: hi^T in rows [0, 64), lo^T in rows
 * [64, 128) (R < 64 leaves zero rows).  Per K-step of 8 rows two MMAs run
 * with M = 128 and N = R rounded up to 16:
 *     D += [hi; lo]^T-rows x hi      and      D += [hi; lo]^T-rows x lo
 * so D[0:64] = hi^T hi + hi^T lo and D[64:128] = lo^T hi + lo^T lo, and
 * G = D[0:64] + D[64:128] = (hi + lo)^T (hi + lo).  The B operand is the
 * same tile (its hi or lo rows), so no second staging is needed.
 *
 * Each CTA (128 threads) owns up to 4096 rows.  The tensor core accumulates
 * in FP32 in TMEM; every 16 chunks (512 rows) the accumulator is drained
 * into FP64 registers (thread t holds TMEM row t) and the next MMA starts a
 * fresh FP32 sum.  At the end the CTA adds its R x R tile into the FP64 G
 * with atomics.  Two stages:
 * threads fill one tile while the tensor core reads the other; a
 * tcgen05.commit per chunk arrives on that stage's mbarrier.  Every mbarrier
 * wait is bounded by a deadline; on expiry the kernel records an error,
 * waits once more (bounded) for its MMAs, frees its TMEM and returns.
 *
 * Shared-memory operand layout: K-major, no swizzle -- core matrices of
 * 8 rows x 16 bytes (4 TF32 values) stored contiguously (128 B); the 16
 * row groups of a K column of core matrices are 128 B apart (SBO) and the
 * K columns 2048 B apart (LBO).  Element (row m, k) of a chunk is at
 * (k / 4) * 2048 + (m / 8) * 128 + (m % 8) * 16 + (k % 4) * 4.
 */
#include "common.cuh"

namespace sb {
namespace {

constexpr int GT_THREADS = 128;
constexpr int GT_KC = 32;                                   /* rows per chunk */
constexpr int GT_M = 128;                                   /* MMA M */
constexpr uint32_t GT_SBO = 128;                            /* 8-row group stride */
constexpr uint32_t GT_LBO = (GT_M / 8) * 128;               /* K core-column stride */
constexpr uint32_t GT_TILE = (uint32_t) GT_KC * GT_M * 4;   /* 16 KB per stage */
constexpr uint32_t GT_LO = 8 * GT_SBO;                      /* lo rows start at m = 64 */
constexpr uint64_t GT_MAX_ROWS_PER_CTA = 4096;
constexpr unsigned long long GT_DEADLINE_NS = 1000000000ull; /* 1 s */
constexpr uint32_t GT_DRAIN = 16;                           /* chunks per FP32 sum */

__device__ __forceinline__ uint32_t smem_u32(void const * p)
{
  return (uint32_t) __cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long gt_now()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

/* shared-memory matrix descriptor: start address, LBO, SBO (16-byte
 * units), version 1, no swizzle */
__device__ __forceinline__ uint64_t gt_desc(uint32_t saddr)
{
  uint64_t d = (uint64_t) ((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t) ((GT_LBO >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t) ((GT_SBO >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t) 1 << 46;
  return d;
}

/* instruction descriptor: D F32, A and B TF32, both K-major, N, M = 128 */
__device__ __forceinline__ uint32_t gt_idesc(uint32_t N)
{
  return (1u << 4) | (2u << 7) | (2u << 10) | ((N >> 3) << 17) | ((uint32_t) (GT_M >> 4) << 24);
}

__device__ __forceinline__ uint32_t tf32_rna(float x)
{
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ bool gt_mbar_wait(uint32_t bar, uint32_t parity)
{
  unsigned long long const t0 = gt_now();
  for(;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done) : "r"(bar), "r"(parity) : "memory");
    if(done) { return true; }
    if(gt_now() - t0 > GT_DEADLINE_NS) { return false; }
  }
}

__device__ __forceinline__ void gt_mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc,
    uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      :: "r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate) : "memory");
}

__global__ void __launch_bounds__(GT_THREADS, 1)
k_gram_tc(float const * __restrict__ A, uint64_t nrows, uint32_t R, uint32_t ld,
    uint64_t rows_per_cta, double * __restrict__ G, int * __restrict__ err)
{
  extern __shared__ __align__(1024) unsigned char gt_smem[];   /* 2 stages */
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t s_tmem;
  uint32_t const tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint64_t const r0 = (uint64_t) blockIdx.x * rows_per_cta;
  if(r0 >= nrows) { return; }                                  /* whole block */
  uint64_t const r1 = umin64(nrows, r0 + rows_per_cta);
  uint32_t const N = R <= 16 ? 16u : ((R + 15u) & ~15u);
  uint32_t const ncols = N <= 32 ? 32u : 64u;

  if(warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(&s_tmem)), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if(tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&mbar[0])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&mbar[1])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  uint32_t const tmem = s_tmem;
  uint32_t const idesc = gt_idesc(N);
  uint32_t const tile0 = smem_u32(gt_smem);
  uint32_t const nchunks = (uint32_t) ((r1 - r0 + GT_KC - 1) / GT_KC);

  bool ok = true;
  int last = -1;                                   /* last chunk committed */
  double acc[64];                                  /* FP64 sums of TMEM row `tid` */
#pragma unroll
  for(int j = 0; j < 64; ++j) { acc[j] = 0.; }
  for(uint32_t c = 0; c < nchunks; ++c) {
    uint32_t const st = c & 1u;
    bool w = true;
    if(c >= 2) { w = gt_mbar_wait(smem_u32(&mbar[st]), ((c >> 1) - 1u) & 1u); }
    if(!__syncthreads_and(w)) { ok = false; break; }
    /* fill: lane (m % 8, k % 4) = (lane % 8, lane / 8): conflict-free stores */
    unsigned char * tile = gt_smem + st * GT_TILE;
    uint64_t const rb = r0 + (uint64_t) c * GT_KC;
#pragma unroll 4
    for(uint32_t it = 0; it < 16; ++it) {
      uint32_t const q = it * 4 + warp;
      uint32_t const m = (q & 7u) * 8 + (lane & 7u);
      uint32_t const k = (q >> 3) * 4 + (lane >> 3);
      uint64_t const row = rb + k;
      float const x = (row < r1 && m < R) ? __ldg(A + row * ld + m) : 0.f;
      uint32_t const hi = tf32_rna(x);
      uint32_t const lo = tf32_rna(x - __uint_as_float(hi));
      uint32_t const off = (k >> 2) * GT_LBO + (m >> 3) * GT_SBO + (m & 7u) * 16 + (k & 3u) * 4;
      *(uint32_t *) (tile + off) = hi;
      *(uint32_t *) (tile + off + GT_LO) = lo;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if(tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      uint32_t const base = tile0 + st * GT_TILE;
#pragma unroll
      for(uint32_t s = 0; s < GT_KC / 8; ++s) {
        uint32_t const kb = base + s * 2 * GT_LBO;
        uint64_t const da = gt_desc(kb);
        gt_mma(tmem, da, da, idesc, (c % GT_DRAIN != 0 || s > 0) ? 1u : 0u);   /* x hi */
        gt_mma(tmem, da, gt_desc(kb + GT_LO), idesc, 1u);           /* x lo */
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   :: "r"(smem_u32(&mbar[st])) : "memory");
    }
    last = (int) c;
    if((c + 1) % GT_DRAIN == 0 || c + 1 == nchunks) {
      /* drain: this chunk's commit tracks every earlier MMA of thread 0 */
      bool const w = gt_mbar_wait(smem_u32(&mbar[st]), (c >> 1) & 1u);
      if(!__syncthreads_and(w)) { ok = false; break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      /* warp w reads TMEM lanes [32w, 32w + 32): row tid of D */
#pragma unroll
      for(uint32_t cb = 0; cb < 64; cb += 16) {
        if(cb >= N) { break; }
        uint32_t v[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
            "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
              "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
              "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(tmem + ((warp * 32u) << 16) + cb));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for(int j = 0; j < 16; ++j) { acc[cb + j] += (double) __uint_as_float(v[j]); }
      }
      /* every lane's loads are done before the next MMA overwrites D */
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
    }
  }
  if(ok && last >= 0) {
    /* rows [0, 64) + rows [64, 128) of the FP64 sums, via shared memory */
    double * D = (double *) gt_smem;               /* 128 x 64 doubles = 64 KB */
#pragma unroll
    for(int j = 0; j < 64; ++j) { D[tid * 64 + j] = acc[j]; }
    __syncthreads();
    for(uint32_t e = tid; e < R * R; e += GT_THREADS) {
      uint32_t const i = e / R, j = e % R;
      if(j < i) { continue; }                      /* upper triangle, as sb_gram */
      atomicAdd(G + e, D[i * 64 + j] + D[(64 + i) * 64 + j]);
    }
  } else if(last >= 0) {
    if(tid == 0) { atomicExch(err, 1); }
    /* a wait expired: give the issued MMAs one more bounded wait before
     * their TMEM is released */
    gt_mbar_wait(smem_u32(&mbar[last & 1]), ((uint32_t) last >> 1) & 1u);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if(warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :: "r"(tmem), "r"(ncols) : "memory");
  }
}

} /* namespace */
} /* namespace sb */

using namespace sb;

extern "C" {

/* G (R x R, double, upper triangle; the lower one is zero) = A^T A for an
 * FP32 A with split TF32 tensor-core products; R <= 64.  G is overwritten. */
int sb_gram_tc(float const * A, uint64_t I, uint32_t R, uint32_t ld, double * G)
{
  if(R == 0 || R > 64 || ld < R) { return SB_EINPUT; }
  SB_TRY(cudaMemsetAsync(G, 0, (size_t) R * R * sizeof(double), stream()));
  if(I == 0) { return SB_OK; }
  /* at most 4096 rows per CTA (FP32 accumulation in TMEM), at least ~4
   * CTAs per SM worth of work when the matrix is large */
  uint64_t nb = (I + GT_MAX_ROWS_PER_CTA - 1) / GT_MAX_ROWS_PER_CTA;
  uint64_t const want = (I + GT_KC - 1) / GT_KC;
  uint64_t const cap = 148 * 4;
  if(nb < cap) { nb = want < cap ? want : cap; }
  uint64_t rows = (I + nb - 1) / nb;
  rows = (rows + GT_KC - 1) / GT_KC * GT_KC;
  nb = (I + rows - 1) / rows;
  int * err = nullptr;
  int rc = talloc(&err, 1);
  if(rc) { return rc; }
  SB_TRY(cudaMemsetAsync(err, 0, sizeof(int), stream()));
  /* two 16 KB stages; the allocation is 64 KB so that every address an
   * operand descriptor can reach (16 row groups x the 2 KB K stride from
   * either stage) stays inside this CTA's shared memory */
  size_t const smem = 4 * (size_t) GT_TILE;
  cudaFuncSetAttribute(k_gram_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
  k_gram_tc<<<(unsigned) nb, GT_THREADS, smem, stream()>>>(A, I, R, ld, rows, G, err);
  cudaError_t const e = cudaGetLastError();
  int herr = 0;
  if(e == cudaSuccess) {
    SB_TRY(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, stream()));
    SB_TRY(cudaStreamSynchronize(stream()));
  }
  tfree(err);
  if(e != cudaSuccess) { return fail(e); }
  return herr ? SB_EDEVICE : SB_OK;
}

} /* extern "C" */
