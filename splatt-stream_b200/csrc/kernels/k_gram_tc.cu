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
 * Each CTA owns a contiguous range of rows (the TMA-fed kernel: two CTAs
 * per SM; the thread-loaded one: at most 4096 rows).  The tensor core accumulates
 * in FP32 in TMEM; every 16 chunks (512 rows) the accumulator is drained
 * into FP64 registers (thread t holds TMEM row t) and the next MMA starts a
 * fresh FP32 sum.  At the end the CTA adds its R x R tile into the FP64 G
 * with atomics.  Two stages:
 * threads fill one tile while the tensor core reads the other; a
 * tcgen05.commit per chunk arrives on that stage's mbarrier.  Every mbarrier
 * wait is bounded by a deadline; on expiry the kernel records an error,
 * waits once more (bounded) for its MMAs, frees its TMEM and returns.
 *
 * Two kernels share that scheme and differ in how rows reach shared memory:
 *
 * k_gram_tc_tma (R a multiple of 4, 16-byte aligned rows): TMA bulk tensor
 * copies of 64-row chunks into a ring of 2 raw stages (one thread issues
 * them; completion on per-stage mbarriers), two CTAs resident per SM so that
 * one CTA's split, MMA issue and drain overlap the other's (one CTA per SM
 * with 6 stages ran at 72% of this rate), viewing A as a 3-D tensor
 * (4 columns, rows, R/4 column groups): a raw stage is [group][row][4].
 * Threads split each element into the K-major hi / lo operand layout
 * below, with the K core-column stride padded by 16 bytes (a warp takes two
 * column groups x 16 rows: conflict-free 16-byte reads of the raw stage
 * and conflict-free stores).
 *
 * k_gram_tc (any R <= 64, any ld): threads load the rows and store them
 * K-major (layout below).
 *
 * K-major operand layout of k_gram_tc: no swizzle -- core matrices of
 * 8 rows x 16 bytes (4 TF32 values) stored contiguously (128 B); the 16
 * row groups of a K column of core matrices are 128 B apart (SBO) and the
 * K columns 2048 B apart (LBO).  Element (row m, k) of a chunk is at
 * (k / 4) * 2048 + (m / 8) * 128 + (m % 8) * 16 + (k % 4) * 4.
 */
#include "common.cuh"
#include <cuda.h>
#include <cudaTypedefs.h>

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
__device__ __forceinline__ uint64_t gt_desc(uint32_t saddr, uint32_t lbo = GT_LBO)
{
  uint64_t d = (uint64_t) ((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t) ((lbo >> 4) & 0x3FFFu) << 16;
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

/* ---- TMA-fed variant ---------------------------------------------------- */
constexpr int GQ_THREADS = 256;                             /* 8 warps split */
constexpr int GQ_KC = 64;                                   /* rows per chunk */
constexpr int GQ_STAGES = 2;                                /* raw TMA stages */
constexpr int GQ_CTAS_PER_SM = 2;                           /* resident CTAs per SM */
constexpr uint32_t GQ_GRP = GQ_KC * 16;                     /* one column group: 1 KB */
constexpr uint32_t GQ_RAW = 16 * GQ_GRP;                    /* 64 columns: 16 KB */
/* K core-column stride of the operand: 16 row groups of 128 B plus 16 B of
 * padding, so that the split's stores (a warp: 16 rows x 2 column groups,
 * one column of each group per store) fall in 32 different banks: the
 * word offset mod 32 is 4 (k / 4) + k % 4 + 16 (g % 2) + 4 x */
constexpr uint32_t GQ_LBO = GT_LBO + 16;
constexpr uint32_t GQ_OP = (GQ_KC / 4) * GQ_LBO;            /* K-major hi + lo: 33 KB */
constexpr uint32_t GQ_DRAIN = 8;                            /* chunks per FP32 sum */
constexpr size_t GQ_SMEM = (size_t) GQ_STAGES * GQ_RAW + 2 * GQ_OP;   /* 98 KB */
static_assert(GQ_OP % 16 == 0 && GQ_CTAS_PER_SM * (GQ_SMEM + 1024) <= 228 * 1024, "operand buffers");

__device__ __forceinline__ void gq_tma(uint32_t dst, CUtensorMap const * tm, int row, uint32_t bar,
    uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               :: "r"(bar), "r"(bytes) : "memory");
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3, %4}], [%5];"
      :: "r"(dst), "l"((uint64_t) tm), "r"(0), "r"(row), "r"(0), "r"(bar) : "memory");
}

__global__ void __launch_bounds__(GQ_THREADS, GQ_CTAS_PER_SM)
k_gram_tc_tma(const __grid_constant__ CUtensorMap tmap, uint64_t nrows, uint32_t R,
    uint64_t rows_per_cta, double * __restrict__ G, int * __restrict__ err)
{
  extern __shared__ __align__(1024) unsigned char gq_smem[];
  __shared__ __align__(8) uint64_t full[GQ_STAGES];
  __shared__ __align__(8) uint64_t mmab[2];
  __shared__ uint32_t s_tmem;
  __shared__ int s_issued;
  uint32_t const tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint64_t const r0 = (uint64_t) blockIdx.x * rows_per_cta;
  if(r0 >= nrows) { return; }                                  /* whole block */
  uint64_t const r1 = umin64(nrows, r0 + rows_per_cta);
  uint32_t const N = R <= 16 ? 16u : ((R + 15u) & ~15u);
  uint32_t const ncols = N <= 32 ? 32u : 64u;
  uint32_t const G4 = R >> 2;                                  /* column groups */
  uint32_t const tx = (uint32_t) GQ_KC * R * 4;                /* bytes per box */
  uint32_t const nchunks = (uint32_t) ((r1 - r0 + GQ_KC - 1) / GQ_KC);
  unsigned char * raw = gq_smem;
  unsigned char * ops = gq_smem + GQ_STAGES * GQ_RAW;

  if(warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(&s_tmem)), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if(tid == 0) {
    for(int i = 0; i < GQ_STAGES; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&full[i])) : "memory");
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&mmab[0])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&mmab[1])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  /* operand buffers start at zero: column groups >= R/4 stay zero */
  for(uint32_t i = tid; i < 2 * GQ_OP / 16; i += GQ_THREADS) {
    ((float4 *) ops)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  uint32_t const tmem = s_tmem;
  uint32_t const idesc = gt_idesc(N);
  if(tid == 0) {
    uint32_t const np = nchunks < (uint32_t) GQ_STAGES ? nchunks : (uint32_t) GQ_STAGES;
    for(uint32_t p = 0; p < np; ++p) {
      gq_tma(smem_u32(raw + p * GQ_RAW), &tmap, (int) (r0 + (uint64_t) p * GQ_KC),
             smem_u32(&full[p]), tx);
    }
    s_issued = (int) np;
  }

  bool ok = true;
  int last = -1;
  /* FP64 sums: warp w holds TMEM lanes [32 (w % 4), +32), columns
   * [32 (w / 4), +32) */
  uint32_t const lane0 = (warp & 3u) * 32u, col0 = (warp >> 2) * 32u;
  double acc[32];
#pragma unroll
  for(int j = 0; j < 32; ++j) { acc[j] = 0.; }
  for(uint32_t c = 0; c < nchunks; ++c) {
    uint32_t const s = c % GQ_STAGES, o = c & 1u;
    bool w = gt_mbar_wait(smem_u32(&full[s]), (c / GQ_STAGES) & 1u);
    if(c >= 2) { w = w && gt_mbar_wait(smem_u32(&mmab[o]), ((c >> 1) - 1u) & 1u); }
    if(!__syncthreads_and(w)) { ok = false; break; }
    /* split the raw stage [group][row][4] into the K-major operand: a warp
     * takes two column groups x 16 rows per step (lane: row = lane % 16,
     * group = lane / 16) */
    float4 const * rs = (float4 const *) (raw + s * GQ_RAW);
    unsigned char * op = ops + o * GQ_OP;
    uint32_t const nunits = ((G4 + 1) >> 1) * (GQ_KC / 16);
    for(uint32_t u = warp; u < nunits; u += GQ_THREADS / 32) {
      uint32_t const g = (u / (GQ_KC / 16)) * 2 + (lane >> 4);
      uint32_t const k = (u % (GQ_KC / 16)) * 16 + (lane & 15u);
      if(g >= G4) { continue; }
      float4 const v = rs[g * GQ_KC + k];
      float const x4[4] = {v.x, v.y, v.z, v.w};
      uint32_t const kb = (k >> 2) * GQ_LBO + (k & 3u) * 4;
#pragma unroll
      for(int x = 0; x < 4; ++x) {
        uint32_t const m = g * 4 + (uint32_t) x;
        uint32_t const off = kb + (m >> 3) * GT_SBO + (m & 7u) * 16;
        uint32_t const hi = tf32_rna(x4[x]);
        *(uint32_t *) (op + off) = hi;
        *(uint32_t *) (op + off + GT_LO) = tf32_rna(x4[x] - __uint_as_float(hi));
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if(tid == 0) {
      if(c + GQ_STAGES < nchunks) {            /* the raw stage is free again */
        uint32_t const cn = c + GQ_STAGES;
        gq_tma(smem_u32(raw + s * GQ_RAW), &tmap, (int) (r0 + (uint64_t) cn * GQ_KC),
               smem_u32(&full[s]), tx);
        s_issued = (int) cn + 1;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      uint32_t const base = smem_u32(ops + o * GQ_OP);
#pragma unroll
      for(uint32_t st = 0; st < GQ_KC / 8; ++st) {
        uint32_t const kb = base + st * 2 * GQ_LBO;
        uint64_t const da = gt_desc(kb, GQ_LBO);
        gt_mma(tmem, da, da, idesc, (c % GQ_DRAIN != 0 || st > 0) ? 1u : 0u);   /* x hi */
        gt_mma(tmem, da, gt_desc(kb + GT_LO, GQ_LBO), idesc, 1u);                /* x lo */
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   :: "r"(smem_u32(&mmab[o])) : "memory");
    }
    last = (int) c;
    if((c + 1) % GQ_DRAIN == 0 || c + 1 == nchunks) {
      bool const wd = gt_mbar_wait(smem_u32(&mmab[o]), (c >> 1) & 1u);
      if(!__syncthreads_and(wd)) { ok = false; break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for(uint32_t cb = 0; cb < 32; cb += 16) {
        if(col0 + cb >= N) { break; }
        uint32_t v[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
            "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
              "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
              "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(tmem + (lane0 << 16) + col0 + cb));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for(int j = 0; j < 16; ++j) { acc[cb + j] += (double) __uint_as_float(v[j]); }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
    }
  }
  if(ok && last >= 0) {
    double * D = (double *) gq_smem;               /* 128 x 64 doubles = 64 KB */
    uint32_t const m = lane0 + lane;
#pragma unroll
    for(int j = 0; j < 32; ++j) { D[m * 64 + col0 + j] = acc[j]; }
    __syncthreads();
    for(uint32_t e = tid; e < R * R; e += GQ_THREADS) {
      uint32_t const i = e / R, j = e % R;
      if(j < i) { continue; }                      /* upper triangle, as sb_gram */
      atomicAdd(G + e, D[i * 64 + j] + D[(64 + i) * 64 + j]);
    }
  } else {
    if(tid == 0) { atomicExch(err, 1); }
    /* a wait expired: give the copies and MMAs in flight one more bounded
     * wait each before the shared memory and TMEM are released */
    __syncthreads();
    int const issued = s_issued;
    for(int c = (last < 0 ? 0 : last + 1); c < issued; ++c) {
      gt_mbar_wait(smem_u32(&full[c % GQ_STAGES]), ((uint32_t) c / GQ_STAGES) & 1u);
    }
    if(last >= 0) { gt_mbar_wait(smem_u32(&mmab[last & 1]), ((uint32_t) last >> 1) & 1u); }
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

/* cuTensorMapEncodeTiled through the runtime's driver entry point (no link
 * against libcuda); NULL when the driver does not provide it */
PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder()
{
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if(!tried) {
    tried = true;
    void * p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess) {
      fn = (PFN_cuTensorMapEncodeTiled_v12000) p;
    }
    cudaGetLastError();
  }
  return fn;
}


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
  PFN_cuTensorMapEncodeTiled_v12000 const enc = tmap_encoder();
  CUtensorMap tm;
  bool tma = enc && R % 4 == 0 && ld % 4 == 0 && ((uintptr_t) A) % 16 == 0 && I < (1ull << 31);
  if(tma) {
    /* A as a 3-D tensor: (4 columns, rows, R/4 column groups) */
    cuuint64_t const dims[3] = {4, (cuuint64_t) I, (cuuint64_t) (R / 4)};
    cuuint64_t const strides[2] = {(cuuint64_t) ld * 4, 16};
    cuuint32_t const box[3] = {4, (cuuint32_t) GQ_KC, (cuuint32_t) (R / 4)};
    cuuint32_t const estr[3] = {1, 1, 1};
    tma = enc(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *) A, dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  }
  if(tma) {
    /* two CTAs per SM, each streaming a contiguous range (the FP32 sums are
     * drained to FP64 every 512 rows, so the range length does not bound
     * the accuracy); rows per CTA a multiple of the 64-row chunk, so boxes
     * never reach into the next CTA's rows */
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    uint64_t nqa = (I + GQ_KC - 1) / GQ_KC;
    if(nqa > (uint64_t) nsm * GQ_CTAS_PER_SM) { nqa = (uint64_t) nsm * GQ_CTAS_PER_SM; }
    uint64_t rq = (I + nqa - 1) / nqa;
    rq = (rq + GQ_KC - 1) / GQ_KC * GQ_KC;
    unsigned const nq = (unsigned) ((I + rq - 1) / rq);
    cudaFuncSetAttribute(k_gram_tc_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) GQ_SMEM);
    k_gram_tc_tma<<<nq, GQ_THREADS, GQ_SMEM, stream()>>>(tm, I, R, rq, G, err);
  } else {
    /* two 16 KB stages; the allocation is 64 KB so that every address an
     * operand descriptor can reach (16 row groups x the 2 KB K stride from
     * either stage) stays inside this CTA's shared memory */
    size_t const smem = 4 * (size_t) GT_TILE;
    cudaFuncSetAttribute(k_gram_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    k_gram_tc<<<(unsigned) nb, GT_THREADS, smem, stream()>>>(A, I, R, ld, rows, G, err);
  }
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
