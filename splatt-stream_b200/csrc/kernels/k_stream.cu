/*
 * k_stream.cu -- the per-slice update of streaming CPD on the device.
 *
 * Replaces StreamCPD::compute's per-batch body (src/cpd/stream/StreamCPD.cc:
 * 378-512): grow_mats' Gram refresh (192-220), the time-row frob solve
 * (admm() closed form, src/cpd/admm.c:217-235 + frob.c:25-37), the temporal
 * Gram update (423-435), per non-streamed mode the COO MTTKRP
 * (src/mttkrp.c:1699-1769), add_historical (223-294), ADMM with the
 * max-column-norm prox (src/cpd/admm.c:240-406, maxcolnorm.c:32-62), the
 * Gram and delta updates (460-470), the outer convergence test (475), the
 * forgetting factor (490-492) and the old<-new copy (497-503).
 *
 * The update is written as a sequence of grid-wide phases.  Each phase is a
 * __device__ function over a "virtual grid" (block vb of nvb); reductions end
 * in the last block to finish (threadfence + counter), so a phase's result is
 * complete when the phase returns everywhere.  Two executors share them:
 *   PLAIN: one launch per phase, the host reads the ADMM / outer convergence
 *          flags between launches (the reference's control flow, FP64);
 *   FUSED: one cooperative persistent launch per slice; phases separated by a
 *          grid barrier whose wait is bounded by a deadline (an expired wait
 *          sets an error flag, every block leaves, the host sees the flag).
 * Data written by another block during a fused launch is read with
 * ld.global.cg (L2) so no block sees a stale L1 line.
 *
 * ADMM solve: each mode update forms (G + rho I) in FP64, factors it
 * (Cholesky, as dpotrf) and forms its inverse from the factor
 * (L^{-T} L^{-1}); every inner iteration then multiplies the auxiliary rows
 * by that R x R matrix -- one row-times-matrix product instead of 2R
 * dependent substitution steps per row.  All Gram, Cholesky, inverse, norm
 * and convergence arithmetic is FP64 in both precisions.
 */
#include "common.cuh"
#include "kstream.h"

namespace sb {

constexpr int ST_THREADS = 512;

/* dynamic shared memory layout (doubles), R = rank:
 *   [0, R^2)            Cholesky scratch S / cross-product staging (64R)
 *   [R^2, 2R^2)         Ginv (persists through a mode's ADMM loop)
 *   [2R^2, 3R^2)        hb   (historical multiplier)
 *   [3R^2, 3R^2+512)    small slots (column sums, norms, rho, ...)
 *   [3R^2+512, +R^2+64) final-reduction buffer
 * staging (64R doubles) only runs in phases where Ginv/hb are dead. */
__host__ __device__ __forceinline__ uint32_t sm_small(uint32_t R) { return 3 * R * R; }
__host__ __device__ __forceinline__ uint32_t sm_big(uint32_t R) { return 3 * R * R + 512; }
/* per-warp staging of 4 auxiliary rows (row stride SB_XS_STRIDE elements)
 * after the final-reduction buffer, 16-byte aligned */
#define SB_XS_STRIDE 64
__host__ __device__ __forceinline__ uint32_t sm_xs(uint32_t R) { return (sm_big(R) + R * R + 64 + 1) & ~1u; }

/* red[] layout (doubles).  Accumulators are filled with FP64 atomics by
 * every block after a shared-memory reduction; a buffer read in one phase is
 * re-zeroed (by block 0) one phase before it is accumulated again, so the
 * ADMM accumulators alternate between two copies by iteration parity. */
enum {
  RD_RHO = 0,                 /* rho of the current mode update */
  RD_CN = 16,                 /* 4 x 64: column sums of P^2, ring by ADMM counter */
  RD_NRM = RD_CN + 256,       /* 4 x 4: dual norm, primal norm, primal/dual residuals */
  RD_DACC = RD_NRM + 16,      /* 2 x 8 x 2: ||Aold - Anew||^2, ||Anew||^2 per mode */
  RD_NACC = RD_DACC + 32,     /* 8 x 64: first-slice column sums of squares */
  RD_SIZE = RD_NACC + 512
};
static_assert(RD_NRM == SB_RD_NRM && RD_DACC == SB_RD_DACC && RD_SIZE <= SB_RED_SIZE,
    "red[] layout shared with the host");

template <typename T>
__device__ __forceinline__ T ldcg(T const * p) { return __ldcg(p); }

__device__ __forceinline__ unsigned long long gtimer()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

/* bounded grid barrier: returns false (in every thread) when the error flag
 * is set or the wait exceeded the deadline */
__device__ bool grid_barrier(unsigned * bar, int * err, unsigned nblocks)
{
  __shared__ int s_ok;
  __syncthreads();
  if(threadIdx.x == 0) {
    volatile unsigned * gen = bar + 1;
    unsigned const g = *gen;
    __threadfence();
    unsigned const a = atomicAdd(bar, 1u);
    int ok = 1;
    if(a == nblocks - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      unsigned long long const t0 = gtimer();
      while(*gen == g) {
        if(*(volatile int *) err) { ok = 0; break; }
        if(gtimer() - t0 > 2000000000ull) {     /* 2 s */
          atomicExch(err, 2);
          ok = 0;
          break;
        }
        __nanosleep(40);
      }
    }
    __threadfence();
    s_ok = ok && (*(volatile int *) err == 0);
  }
  __syncthreads();
  return s_ok != 0;
}

__device__ __forceinline__ void row_range(uint32_t n, unsigned vb, unsigned nvb, uint32_t & r0,
    uint32_t & r1)
{
  uint64_t const a = (uint64_t) n * vb / nvb;
  uint64_t const b = (uint64_t) n * (vb + 1) / nvb;
  r0 = (uint32_t) a;
  r1 = (uint32_t) b;
}

/* dst(i,j) += sum over rows [r0, r1) of X[r][i] * Y[r][j]  (R x R, full),
 * one FP64 atomic per entry per block.  X, Y: T rows; sh stages 2 x 32 rows. */
template <typename T>
__device__ void block_cross_add(T const * X, T const * Y, uint32_t r0, uint32_t r1, uint32_t R,
    double * dst, double * sh)
{
  uint32_t const npairs = R * R;
  /* R <= 64 and blockDim = 512: at most 8 (i, j) pairs per thread */
  double acc[8] = {0., 0., 0., 0., 0., 0., 0., 0.};
  for(uint32_t rb = r0; rb < r1; rb += 32) {
    uint32_t const nr = umin32(32, r1 - rb);
    __syncthreads();
    {
      uint32_t const lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
      for(uint32_t rr = w; rr < nr; rr += nw) {
        for(uint32_t c = lane; c < R; c += 32) {
          sh[rr * R + c] = (double) ldcg(X + (size_t) (rb + rr) * R + c);
          sh[32 * R + rr * R + c] = (double) ldcg(Y + (size_t) (rb + rr) * R + c);
        }
      }
    }
    __syncthreads();
#pragma unroll
    for(int q = 0; q < 8; ++q) {
      uint32_t const p = threadIdx.x + (uint32_t) q * blockDim.x;
      if(p < npairs) {
        uint32_t const i = p / R, j = p % R;
        double s = acc[q];
        for(uint32_t rr = 0; rr < nr; ++rr) { s = fma(sh[rr * R + i], sh[32 * R + rr * R + j], s); }
        acc[q] = s;
      }
    }
  }
  if(r1 > r0) {
#pragma unroll
    for(int q = 0; q < 8; ++q) {
      uint32_t const p = threadIdx.x + (uint32_t) q * blockDim.x;
      if(p < npairs) { atomicAdd(dst + p, acc[q]); }
    }
  }
  __syncthreads();
}

/* block-reduce `n` (<= 64) per-thread column values held by lanes (col c of
 * warp w) into global accumulators with one atomic per column per block */
__device__ void block_cols_add(double * sh, uint32_t R, uint32_t c0, double v0, double v1,
    bool ok0, bool ok1, double * dst)
{
  __syncthreads();
  for(uint32_t c = threadIdx.x; c < R; c += blockDim.x) { sh[c] = 0.; }
  __syncthreads();
  if(ok0) { atomicAdd(&sh[c0], v0); }
  if(ok1) { atomicAdd(&sh[c0 + 32], v1); }
  __syncthreads();
  for(uint32_t c = threadIdx.x; c < R; c += blockDim.x) { atomicAdd(dst + c, sh[c]); }
}

/* In-block FP64 Cholesky of S (R x R full symmetric in smem, lower used);
 * returns the first bad pivot + 1 (0 if positive definite). */
__device__ int block_cholesky(double * S, uint32_t R)
{
  __shared__ int s_bad;
  if(threadIdx.x == 0) { s_bad = 0; }
  __syncthreads();
  for(uint32_t k = 0; k < R; ++k) {
    if(threadIdx.x == 0) {
      double const d = S[k * R + k];
      if(!(d > 0.) && s_bad == 0) { s_bad = (int) k + 1; }
      S[k * R + k] = sqrt(d > 0. ? d : 1.);
    }
    __syncthreads();
    double const piv = S[k * R + k];
    for(uint32_t i = k + 1 + threadIdx.x; i < R; i += blockDim.x) { S[i * R + k] /= piv; }
    __syncthreads();
    uint32_t const w = R - k - 1;
    for(uint32_t e = threadIdx.x; e < w * w; e += blockDim.x) {
      uint32_t const i = k + 1 + e / w, j = k + 1 + e % w;
      if(j <= i) { S[i * R + j] -= S[i * R + k] * S[j * R + k]; }
    }
    __syncthreads();
  }
  return s_bad;
}

/* Given the Cholesky factor L in the lower triangle of S, write the inverse
 * of the original matrix, L^{-T} L^{-1}, to Ginv (R x R full).  X = L^{-1} is
 * built in `X` (R x R scratch) by column-parallel forward substitution: step
 * i finalises row i of X for every column, then updates the rows below. */
__device__ void block_chol_inverse(double const * S, uint32_t R, double * X, double * Ginv)
{
  for(uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) {
    X[e] = (e / R == e % R) ? 1. : 0.;
  }
  __syncthreads();
  for(uint32_t i = 0; i < R; ++i) {
    double const d = S[i * R + i];
    for(uint32_t c = threadIdx.x; c <= i; c += blockDim.x) { X[i * R + c] /= d; }
    __syncthreads();
    uint32_t const w = R - i - 1;
    for(uint32_t e = threadIdx.x; e < w * (i + 1); e += blockDim.x) {
      uint32_t const k = i + 1 + e / (i + 1), c = e % (i + 1);
      X[k * R + c] -= S[k * R + i] * X[i * R + c];
    }
    __syncthreads();
  }
  /* Ginv = X^T X (X lower triangular) */
  for(uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) {
    uint32_t const i = e / R, j = e % R;
    uint32_t const k0 = i > j ? i : j;
    double acc = 0.;
    for(uint32_t k = k0; k < R; ++k) { acc = fma(X[k * R + i], X[k * R + j], acc); }
    Ginv[e] = acc;
  }
  __syncthreads();
}

/* b <- (L L^T)^{-1} b for one vector, L in the lower triangle of S */
__device__ void block_chol_solve_vec(double const * S, uint32_t R, double * b)
{
  for(uint32_t i = 0; i < R; ++i) {
    if(threadIdx.x == 0) { b[i] /= S[i * R + i]; }
    __syncthreads();
    double const yi = b[i];
    for(uint32_t k = i + 1 + threadIdx.x; k < R; k += blockDim.x) { b[k] -= S[k * R + i] * yi; }
    __syncthreads();
  }
  for(uint32_t ii = R; ii-- > 0; ) {
    if(threadIdx.x == 0) { b[ii] /= S[ii * R + ii]; }
    __syncthreads();
    double const xi = b[ii];
    for(uint32_t k = threadIdx.x; k < ii; k += blockDim.x) { b[k] -= S[ii * R + k] * xi; }
    __syncthreads();
  }
}

/* ------------------------------------------------------------------------ */
/* phases                                                                    */
/* ------------------------------------------------------------------------ */
template <typename T>
struct Ph {
  StreamArgs const & a;
  unsigned vb, nvb;
  double * sm;      /* dynamic shared memory */

  __device__ T * A(int m) const { return (T *) a.Anew[m]; }
  __device__ T * Ao(int m) const { return (T *) a.Aold[m]; }
  __device__ T * Dm(int m) const { return (T *) a.D[m]; }
  __device__ T * M() const { return (T *) a.M; }
  __device__ T * AUX() const { return (T *) a.aux; }
  __device__ T * INIT() const { return (T *) a.init; }
  /* ADMM accumulators form a ring of 4 indexed by the slice's ADMM counter k:
   * the phase that accumulates cn(k) clears cn(k+1) and nrm(k+1), whose
   * previous users (k-3) finished at least two grid barriers earlier */
  __device__ double * cn_acc(int k) const { return a.red + RD_CN + (k & 3) * 64; }
  __device__ double * nrm_acc(int k) const { return a.red + RD_NRM + (k & 3) * 4; }
  __device__ double * dacc(int outer, int q) const { return a.red + RD_DACC + (outer & 1) * 16 + 2 * q; }

  /* clear what the slice's phases accumulate into (group block 0) */
  __device__ void clear_accumulators()
  {
    if(vb != 0) { return; }
    uint32_t const R = a.R;
    for(uint32_t e = threadIdx.x; e < SB_RED_SIZE; e += blockDim.x) { a.red[e] = 0.; }
    for(uint32_t c = threadIdx.x; c < R; c += blockDim.x) { a.Mt[c] = 0.; }
    int const nh = a.nns > 1 ? a.nns - 1 : 1;
    for(uint32_t e = threadIdx.x; e < (uint32_t) nh * R * R; e += blockDim.x) { a.H[e] = 0.; }
    for(int q = 0; q < a.nns; ++q) {
      for(uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) { a.G[a.ns[q]][e] = 0.; }
    }
  }

  /* ---- first-slice normalisation: column sums of squares ---- */
  __device__ void colnorm_partial(int q)
  {
    int const m = a.ns[q];
    uint32_t const R = a.R;
    uint32_t r0, r1;
    row_range(a.rows[m], vb, nvb, r0, r1);
    int const lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t const c0 = (uint32_t) lane;
    double v0 = 0., v1 = 0.;
    for(uint32_t i = r0 + w; i < r1; i += nw) {
      if(c0 < R) { double const x = (double) A(m)[(size_t) i * R + c0]; v0 = fma(x, x, v0); }
      if(c0 + 32 < R) { double const x = (double) A(m)[(size_t) i * R + c0 + 32]; v1 = fma(x, x, v1); }
    }
    block_cols_add(sm, R, c0, v0, v1, c0 < R, c0 + 32 < R, a.red + RD_NACC + 64 * q);
  }

  __device__ void colnorm_apply(int q)
  {
    int const m = a.ns[q];
    uint32_t const R = a.R;
    uint32_t r0, r1;
    row_range(a.rows[m], vb, nvb, r0, r1);
    double * nrm = sm;
    for(uint32_t c = threadIdx.x; c < R; c += blockDim.x) {
      nrm[c] = sqrt(ldcg(a.red + RD_NACC + 64 * q + c));
    }
    __syncthreads();
    int const lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for(uint32_t i = r0 + w; i < r1; i += nw) {
      for(uint32_t c = (uint32_t) lane; c < R; c += 32) {
        A(m)[(size_t) i * R + c] = (T) ((double) A(m)[(size_t) i * R + c] / nrm[c]);
      }
    }
  }

  /* ---- Gram of Anew[m] into G[m] (zeroed beforehand) ---- */
  __device__ void gram(int q)
  {
    int const m = a.ns[q];
    uint32_t r0, r1;
    row_range(a.rows[m], vb, nvb, r0, r1);
    block_cross_add<T>(A(m), A(m), r0, r1, a.R, a.G[m], sm);
  }

  /* zero M rows [0, rows) with the virtual grid */
  __device__ void zero_M(uint32_t rows)
  {
    uint64_t const n = (uint64_t) rows * a.R;
    uint64_t const chunk = (n + nvb - 1) / nvb;
    uint64_t const e0 = chunk * vb, e1 = umin64(n, e0 + chunk);
    for(uint64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x) { M()[e] = (T) 0; }
  }

  /* ---- time-mode MTTKRP: Mt[r] += sum_n v prod_{m != sm} A_m[i_m][r];
   * also zeroes M for the first mode ---- */
  __device__ void time_mttkrp(uint32_t zero_rows)
  {
    zero_M(zero_rows);
    uint32_t const R = a.R;
    uint32_t n0, n1;
    row_range(a.nnz, vb, nvb, n0, n1);
    int const lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    T const * vals = (T const *) a.vals;
    double v[2] = {0., 0.};
#pragma unroll
    for(int h = 0; h < 2; ++h) {
      uint32_t const c = (uint32_t) (h * 32 + lane);
      if(h * 32 >= (int) R) { continue; }
      T acc = (T) 0;
      for(uint32_t n = n0 + w; n < n1; n += nw) {
        T p = __ldg(vals + n);
        for(int q = 0; q < a.nns; ++q) {
          int const m = a.ns[q];
          uint32_t const id = __ldg(a.inds[m] + n);
          p *= (c < R) ? ldcg(A(m) + (size_t) id * R + c) : (T) 0;
        }
        acc += p;
      }
      v[h] = (double) acc;
    }
    block_cols_add(sm, R, (uint32_t) lane, v[0], v[1], (uint32_t) lane < R,
        (uint32_t) lane + 32 < R, a.Mt);
  }

  /* ---- time row: s = (Hadamard_{m != sm} G_m + reg I)^{-1} Mt; temporal
   * Gram: mirror, save old, add s s^T (block 0 only) ---- */
  __device__ void time_solve()
  {
    uint32_t const R = a.R;
    if(vb != 0) { return; }
    double * S = sm;
    for(uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) {
      uint32_t const i = e / R, j = e % R;
      uint32_t const u = i < j ? i * R + j : j * R + i;
      double g = 1.;
      for(int q = 0; q < a.nns; ++q) { g *= ldcg(a.G[a.ns[q]] + u); }
      S[e] = g + ((i == j) ? a.reg : 0.);
    }
    __syncthreads();
    int bad = block_cholesky(S, R);
    if(threadIdx.x == 0 && bad) { atomicMax(a.status + 1, bad); }
    double * y = sm + sm_small(R);
    for(uint32_t c = threadIdx.x; c < R; c += blockDim.x) { y[c] = ldcg(a.Mt + c); }
    __syncthreads();
    block_chol_solve_vec(S, R, y);
    double * Gt = a.G[a.sm];
    for(uint32_t c = threadIdx.x; c < R; c += blockDim.x) {
      a.s[c] = y[c];
      ((T *) a.sT)[c] = (T) y[c];
    }
    double * ng = sm + 2 * R * R;
    for(uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) {
      uint32_t const i = e / R, j = e % R;
      /* mirror the upper triangle (p_copy_upper_tri), save, add s s^T */
      double const g = (j >= i) ? Gt[e] : Gt[j * R + i];
      a.old_gram[e] = g;
      ng[e] = g + y[i] * y[j];
    }
    __syncthreads();
    for(uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) { Gt[e] = ng[e]; }
  }

  /* ---- mode MTTKRP (COO, runs of equal output row flushed by atomics) and
   * the historical cross Grams H_o += Aold_o^T Anew_o (o != m, sm).  Block 0
   * clears Mt and the next outer iteration's delta accumulators. ---- */
  __device__ void mode_mttkrp_hist(int mq, int outer)
  {
    int const m = a.ns[mq];
    uint32_t const R = a.R;
    if(mq == 0 && vb == 0) {
      for(uint32_t c = threadIdx.x; c < R; c += blockDim.x) { a.Mt[c] = 0.; }
      for(uint32_t j = threadIdx.x; j < 16; j += blockDim.x) { a.red[RD_DACC + ((outer + 1) & 1) * 16 + j] = 0.; }
    }
    uint32_t n0, n1;
    row_range(a.nnz, vb, nvb, n0, n1);
    int const lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t const per = (n1 - n0 + nw - 1) / nw;
    uint32_t const w0 = n0 + per * w, w1 = umin32(n1, w0 + per);
    T const * vals = (T const *) a.vals;
    uint32_t const * oind = a.inds[m];
    for(uint32_t c0 = 0; c0 < R; c0 += 32) {
      uint32_t const c = c0 + lane;
      T acc = (T) 0;
      uint32_t run = 0xffffffffu;
      for(uint32_t n = w0; n < w1; ++n) {
        uint32_t const o = __ldg(oind + n);
        if(o != run) {
          if(run != 0xffffffffu && c < R) { atomicAdd(M() + (size_t) run * R + c, acc); }
          acc = (T) 0;
          run = o;
        }
        T p = __ldg(vals + n);
        for(int q = 0; q < a.nns; ++q) {
          int const k = a.ns[q];
          if(k == m) { continue; }
          uint32_t const id = __ldg(a.inds[k] + n);
          p *= (c < R) ? ldcg(A(k) + (size_t) id * R + c) : (T) 0;
        }
        /* the time factor row (slice index 0) */
        p *= (c < R) ? ldcg((T const *) a.sT + c) : (T) 0;
        acc += p;
      }
      if(run != 0xffffffffu && c < R) { atomicAdd(M() + (size_t) run * R + c, acc); }
    }
    /* historical cross Grams (H zeroed by the previous mode_finish) */
    int hq = 0;
    for(int q = 0; q < a.nns; ++q) {
      int const o = a.ns[q];
      if(o == m) { continue; }
      uint32_t r0, r1;
      row_range(a.rows[o], vb, nvb, r0, r1);
      block_cross_add<T>(Ao(o), A(o), r0, r1, R, a.H + (size_t) hq * R * R, sm);
      ++hq;
    }
  }

  /* build Ginv = (Hadamard_{k != m} G_k + rho I)^{-1} and the historical
   * multiplier hb = sym(old_gram) o prod_o H_o in shared memory */
  __device__ void mode_setup(int mq, double * Ginv, double * hb)
  {
    int const m = a.ns[mq];
    uint32_t const R = a.R;
    double * S = sm;       /* R*R */
    for(uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) {
      uint32_t const i = e / R, j = e % R;
      uint32_t const u = i < j ? i * R + j : j * R + i;
      double g = 1.;
      for(int k = 0; k < a.N; ++k) { if(k != m) { g *= ldcg(a.G[k] + u); } }
      S[e] = g;
      double h = ldcg(a.old_gram + u);
      int const nh = a.nns - 1;
      for(int q = 0; q < nh; ++q) { h *= ldcg(a.H + (size_t) q * R * R + e); }
      hb[e] = h;
    }
    __syncthreads();
    __shared__ double s_rho;
    if(threadIdx.x == 0) {
      double tr = 0.;
      for(uint32_t i = 0; i < R; ++i) { tr += S[i * R + i]; }
      s_rho = tr / (double) R;
    }
    __syncthreads();
    for(uint32_t i = threadIdx.x; i < R; i += blockDim.x) { S[i * R + i] += s_rho; }
    __syncthreads();
    int const bad = block_cholesky(S, R);
    if(threadIdx.x == 0 && bad && vb == 0) { atomicMax(a.status + 1, bad); }
    block_chol_inverse(S, R, sm + sm_big(R), Ginv);
    if(vb == 0) {
      for(uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) { a.Ginv[e] = Ginv[e]; }
      if(threadIdx.x == 0) { a.red[RD_RHO] = s_rho; }
    }
    sm[sm_small(R) + 500] = s_rho;   /* block-local copy for admm_first */
    __syncthreads();
  }

  /* one row: out = x * Ginv (x in registers, lane holds cols lane, lane+32) */
  __device__ __forceinline__ void row_apply(double const * Ginv, uint32_t R, double x0,
      double x1, double & y0, double & y1)
  {
    int const lane = threadIdx.x & 31;
    double a0 = 0., a1 = 0., b0 = 0., b1 = 0.;
    uint32_t const c0 = (uint32_t) lane, c1 = (uint32_t) lane + 32;
    bool const ok0 = c0 < R, ok1 = c1 < R;
    for(uint32_t k = 0; k < R; k += 2) {
      double const xk = __shfl_sync(0xffffffffu, k < 32 ? x0 : x1, (int) (k & 31));
      double const xl = __shfl_sync(0xffffffffu, k + 1 < 32 ? x0 : x1, (int) ((k + 1) & 31));
      bool const has1 = k + 1 < R;
      if(ok0) {
        a0 = fma(xk, Ginv[k * R + c0], a0);
        if(has1) { b0 = fma(xl, Ginv[(k + 1) * R + c0], b0); }
      }
      if(ok1) {
        a1 = fma(xk, Ginv[k * R + c1], a1);
        if(has1) { b1 = fma(xl, Ginv[(k + 1) * R + c1], b1); }
      }
    }
    y0 = a0 + b0;
    y1 = a1 + b1;
  }

  /* ADMM first half for this block's rows: (first: M += Aold hb, D = 0),
   * init = P, aux = (M + rho (P + D)) Ginv, P = aux - D, column sums of P^2
   * into cn_acc(k); block 0 clears cn_acc(k+1) (and G[m] on the first). */
  __device__ void admm_first(int mq, bool first, int k, double const * Ginv, double const * hb,
      double rho)
  {
    int const m = a.ns[mq];
    uint32_t const R = a.R;
    if(vb == 0) {
      for(uint32_t c = threadIdx.x; c < 64; c += blockDim.x) { cn_acc(k + 1)[c] = 0.; }
      if(threadIdx.x < 4) { nrm_acc(k + 1)[threadIdx.x] = 0.; }
      if(first) {
        for(uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) { a.G[m][e] = 0.; }
      }
    }
    uint32_t r0, r1;
    row_range(a.rows[m], vb, nvb, r0, r1);
    int const lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t const c0 = (uint32_t) lane, c1 = (uint32_t) lane + 32;
    bool const ok0 = c0 < R, ok1 = c1 < R;
    double cs0 = 0., cs1 = 0.;
    T * P = A(m);
    T * D = Dm(m);
    T * Mb = M();
    for(uint32_t i = r0 + w; i < r1; i += nw) {
      size_t const b = (size_t) i * R;
      /* M rows were accumulated by other blocks' atomics: read through L2 */
      double m0 = ok0 ? (double) ldcg(Mb + b + c0) : 0., m1 = ok1 ? (double) ldcg(Mb + b + c1) : 0.;
      double d0 = 0., d1 = 0.;
      if(first) {
        /* M += Aold[i] * hb  (add_historical, StreamCPD.cc:274-291) */
        double o0 = ok0 ? (double) Ao(m)[b + c0] : 0.;
        double o1 = ok1 ? (double) Ao(m)[b + c1] : 0.;
        double h0, h1;
        row_apply(hb, R, o0, o1, h0, h1);
        m0 = (double) (T) (m0 + h0);
        m1 = (double) (T) (m1 + h1);
        if(ok0) { Mb[b + c0] = (T) m0; D[b + c0] = (T) 0; }
        if(ok1) { Mb[b + c1] = (T) m1; D[b + c1] = (T) 0; }
      } else {
        d0 = ok0 ? (double) D[b + c0] : 0.;
        d1 = ok1 ? (double) D[b + c1] : 0.;
      }
      double const p0 = ok0 ? (double) P[b + c0] : 0., p1 = ok1 ? (double) P[b + c1] : 0.;
      if(ok0) { INIT()[b + c0] = (T) p0; }
      if(ok1) { INIT()[b + c1] = (T) p1; }
      /* the reference's auxiliary: M + rho (P + D)  (src/cpd/admm.c:51) */
      double const x0 = (double) (T) (m0 + rho * (p0 + d0));
      double const x1 = (double) (T) (m1 + rho * (p1 + d1));
      double y0, y1;
      row_apply(Ginv, R, x0, x1, y0, y1);
      T const aux0 = (T) y0, aux1 = (T) y1;
      T const np0 = (T) ((double) aux0 - d0), np1 = (T) ((double) aux1 - d1);
      if(ok0) { AUX()[b + c0] = aux0; P[b + c0] = np0; cs0 = fma((double) np0, (double) np0, cs0); }
      if(ok1) { AUX()[b + c1] = aux1; P[b + c1] = np1; cs1 = fma((double) np1, (double) np1, cs1); }
    }
    block_cols_add(sm + sm_small(R), R, c0, cs0, cs1, ok0, ok1, cn_acc(k));
  }

  /* ADMM second half: prox (columns with norm > 1 scaled to unit norm),
   * D += P - aux, the four norms into nrm_acc(k) */
  __device__ void admm_second(int mq, int k)
  {
    int const m = a.ns[mq];
    uint32_t const R = a.R;
    uint32_t r0, r1;
    row_range(a.rows[m], vb, nvb, r0, r1);
    double * cn = sm + sm_small(R) + 128;
    for(uint32_t c = threadIdx.x; c < R; c += blockDim.x) { cn[c] = sqrt(ldcg(cn_acc(k) + c)); }
    __syncthreads();
    double dn = 0., pn = 0., pr = 0., dr = 0.;
    T * P = A(m);
    T * D = Dm(m);
    for(uint64_t e = (uint64_t) r0 * R + threadIdx.x; e < (uint64_t) r1 * R; e += blockDim.x) {
      uint32_t const c = (uint32_t) (e % R);
      double p = (double) P[e];
      if(cn[c] > 1.) { p = (double) (T) (p / cn[c]); P[e] = (T) p; }
      double const au = (double) AUX()[e];
      double const d = (double) (T) ((double) D[e] + p - au);
      D[e] = (T) d;
      dn = fma(d, d, dn);
      double const pd = p - au, dd = p - (double) INIT()[e];
      pn = fma(p, p, pn);
      pr = fma(pd, pd, pr);
      dr = fma(dd, dd, dr);
    }
    dn = warp_sum(dn); pn = warp_sum(pn); pr = warp_sum(pr); dr = warp_sum(dr);
    double * s = sm + sm_small(R) + 256;
    __syncthreads();
    if(threadIdx.x < 4) { s[threadIdx.x] = 0.; }
    __syncthreads();
    if((threadIdx.x & 31) == 0) {
      atomicAdd(&s[0], dn); atomicAdd(&s[1], pn); atomicAdd(&s[2], pr); atomicAdd(&s[3], dr);
    }
    __syncthreads();
    if(threadIdx.x < 4) { atomicAdd(nrm_acc(k) + threadIdx.x, s[threadIdx.x]); }
  }

  /* One pass over this block's rows per ADMM iteration (the fused path):
   * the second half of iteration k (prox with cn(k), D += P - aux, the four
   * norms into nrm(k)) and, when `spec`, the first half of iteration k+1
   * (init = P, aux = (M + rho (P + D)) Ginv, P = aux - D, column sums into
   * cn(k+1)).  Block 0 clears cn(k+2) and nrm(k+2) when it accumulates
   * cn(k+1).
   *
   * Each warp takes four rows at a time.  Their auxiliary inputs x are
   * staged in the warp's shared-memory slice and the row-times-(G + rho I)^-1
   * product reads them back with broadcast vector loads, so one load of an
   * inverse element serves four rows (FP64), or the inverse's column stays
   * in registers (FP32, R <= 32). */
  __device__ void admm_step(int mq, int k, bool spec, double const * Ginv, double rho)
  {
    int const m = a.ns[mq];
    uint32_t const R = a.R;
    if(spec && vb == 0) {
      for(uint32_t c = threadIdx.x; c < 64; c += blockDim.x) { cn_acc(k + 2)[c] = 0.; }
      if(threadIdx.x < 4) { nrm_acc(k + 2)[threadIdx.x] = 0.; }
    }
    double * cn = sm + sm_small(R) + 128;
    for(uint32_t c = threadIdx.x; c < R; c += blockDim.x) { cn[c] = sqrt(ldcg(cn_acc(k) + c)); }
    __syncthreads();
    uint32_t r0, r1;
    row_range(a.rows[m], vb, nvb, r0, r1);
    int const lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t const c0 = (uint32_t) lane, c1 = (uint32_t) lane + 32;
    bool const ok0 = c0 < R, ok1 = c1 < R;
    double const cn0 = ok0 ? cn[c0] : 0., cn1 = ok1 ? cn[c1] : 0.;
    T * xs = (T *) (sm + sm_xs(R)) + (size_t) w * 4 * SB_XS_STRIDE;   /* this warp's 4 rows */
    /* FP32 with R <= 32: the inverse's column c0 in registers */
    constexpr bool REG = sizeof(T) == 4;
    float gcol[32];
    if(REG) {
#pragma unroll
      for(int q = 0; q < 32; ++q) { gcol[q] = ((uint32_t) q < R && ok0) ? (float) Ginv[q * R + c0] : 0.f; }
    }
    bool const use_reg = REG && R <= 32;
    double dn = 0., pn = 0., pr = 0., dr = 0., cs0 = 0., cs1 = 0.;
    T * P = A(m);
    T * D = Dm(m);
    T * AU = AUX();
    T * IN = INIT();
    T const * Mb = M();
    for(uint32_t i0 = r0 + 4 * w; i0 < r1; i0 += 4 * nw) {
      uint32_t const nr = umin32(4, r1 - i0);
      /* second half of iteration k, row by row; stage x for the apply */
      for(uint32_t rr = 0; rr < nr; ++rr) {
        size_t const b = (size_t) (i0 + rr) * R;
#pragma unroll
        for(int h = 0; h < 2; ++h) {
          uint32_t const c = h ? c1 : c0;
          if(!(h ? ok1 : ok0)) { continue; }
          double const cnc = h ? cn1 : cn0;
          double p = (double) P[b + c];
          if(cnc > 1.) { p = (double) (T) (p / cnc); }
          double const au = (double) AU[b + c];
          double const d = (double) (T) ((double) D[b + c] + p - au);
          double const pd = p - au, dd = p - (double) IN[b + c];
          dn = fma(d, d, dn); pn = fma(p, p, pn); pr = fma(pd, pd, pr); dr = fma(dd, dd, dr);
          if(!spec) {
            P[b + c] = (T) p;
            D[b + c] = (T) d;
          } else {
            IN[b + c] = (T) p;
            D[b + c] = (T) d;
            xs[rr * SB_XS_STRIDE + c] = (T) ((double) ldcg(Mb + b + c) + rho * (p + d));
          }
        }
      }
      if(!spec) { continue; }
      for(uint32_t rr = nr; rr < 4; ++rr) {       /* zero the unused staged rows */
        if(ok0) { xs[rr * SB_XS_STRIDE + c0] = (T) 0; }
        if(ok1) { xs[rr * SB_XS_STRIDE + c1] = (T) 0; }
      }
      __syncwarp();
      /* y[rr][c] = sum_q x[rr][q] * Ginv[q][c] */
      double y0[4] = {0., 0., 0., 0.}, y1[4] = {0., 0., 0., 0.};
      if(use_reg) {
        float const * xf = (float const *) xs;
#pragma unroll
        for(int q = 0; q < 32; q += 4) {
          if((uint32_t) q >= R) { break; }
#pragma unroll
          for(int rr = 0; rr < 4; ++rr) {
            float4 const xx = *(float4 const *) (xf + rr * SB_XS_STRIDE + q);
            float acc = 0.f;
            acc = fmaf(xx.x, gcol[q], acc);
            acc = fmaf(xx.y, gcol[q + 1], acc);
            acc = fmaf(xx.z, gcol[q + 2], acc);
            acc = fmaf(xx.w, gcol[q + 3], acc);
            y0[rr] += (double) acc;
          }
        }
      } else {
        for(uint32_t q = 0; q < R; q += 2) {
          bool const two = q + 1 < R;
          double const g00 = ok0 ? Ginv[q * R + c0] : 0.;
          double const g10 = (ok0 && two) ? Ginv[(q + 1) * R + c0] : 0.;
          double const g01 = ok1 ? Ginv[q * R + c1] : 0.;
          double const g11 = (ok1 && two) ? Ginv[(q + 1) * R + c1] : 0.;
#pragma unroll
          for(int rr = 0; rr < 4; ++rr) {
            double xa, xb;
            if(sizeof(T) == 8) {
              double2 const xx = *(double2 const *) ((double const *) xs + rr * SB_XS_STRIDE + q);
              xa = xx.x; xb = xx.y;
            } else {
              float2 const xx = *(float2 const *) ((float const *) xs + rr * SB_XS_STRIDE + q);
              xa = xx.x; xb = xx.y;
            }
            if(!two) { xb = 0.; }
            y0[rr] = fma(xa, g00, fma(xb, g10, y0[rr]));
            y1[rr] = fma(xa, g01, fma(xb, g11, y1[rr]));
          }
        }
      }
      __syncwarp();
      /* first half of iteration k+1: aux = y, P = aux - D */
#pragma unroll
      for(int rr = 0; rr < 4; ++rr) {
        if((uint32_t) rr >= nr) { break; }
        size_t const b = (size_t) (i0 + rr) * R;
        if(ok0) {
          T const au = (T) y0[rr];
          T const np = (T) ((double) au - (double) D[b + c0]);
          AU[b + c0] = au;
          P[b + c0] = np;
          cs0 = fma((double) np, (double) np, cs0);
        }
        if(ok1) {
          T const au = (T) y1[rr];
          T const np = (T) ((double) au - (double) D[b + c1]);
          AU[b + c1] = au;
          P[b + c1] = np;
          cs1 = fma((double) np, (double) np, cs1);
        }
      }
    }
    /* the four norms of iteration k */
    dn = warp_sum(dn); pn = warp_sum(pn); pr = warp_sum(pr); dr = warp_sum(dr);
    double * s = sm + sm_small(R) + 256;
    __syncthreads();
    if(threadIdx.x < 4) { s[threadIdx.x] = 0.; }
    __syncthreads();
    if(lane == 0) {
      atomicAdd(&s[0], dn); atomicAdd(&s[1], pn); atomicAdd(&s[2], pr); atomicAdd(&s[3], dr);
    }
    __syncthreads();
    if(threadIdx.x < 4) { atomicAdd(nrm_acc(k) + threadIdx.x, s[threadIdx.x]); }
    if(spec) { block_cols_add(sm + sm_small(R), R, c0, cs0, cs1, ok0, ok1, cn_acc(k + 1)); }
  }

  /* undo a speculative first half: P back to its value after the second
   * half of the converged iteration (saved in init by the first half) */
  __device__ void admm_rollback(int mq)
  {
    int const m = a.ns[mq];
    uint32_t const R = a.R;
    uint32_t r0, r1;
    row_range(a.rows[m], vb, nvb, r0, r1);
    int const lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for(uint32_t i = r0 + w; i < r1; i += nw) {
      for(uint32_t c = (uint32_t) lane; c < R; c += 32) {
        A(m)[(size_t) i * R + c] = INIT()[(size_t) i * R + c];
      }
    }
  }

  /* the reference's ADMM stopping test (src/cpd/admm.c:300-301) */
  __device__ bool admm_converged(int k) const
  {
    double const dn = ldcg(nrm_acc(k) + 0), pn = ldcg(nrm_acc(k) + 1);
    double const pr = ldcg(nrm_acc(k) + 2), dr = ldcg(nrm_acc(k) + 3);
    return (pr <= a.inner_tol * pn) && (dr <= a.inner_tol * dn);
  }

  /* after ADMM: G[m] += Anew^T Anew (zeroed in the first ADMM phase),
   * ||Aold - Anew||^2, ||Anew||^2 into dacc; block 0 clears H; zero M for
   * the next mode */
  __device__ void mode_finish(int mq, int outer, uint32_t next_rows)
  {
    int const m = a.ns[mq];
    uint32_t const R = a.R;
    if(vb == 0) {
      int const nh = a.nns > 1 ? a.nns - 1 : 1;
      for(uint32_t e = threadIdx.x; e < (uint32_t) nh * R * R; e += blockDim.x) { a.H[e] = 0.; }
    }
    uint32_t r0, r1;
    row_range(a.rows[m], vb, nvb, r0, r1);
    block_cross_add<T>(A(m), A(m), r0, r1, R, a.G[m], sm);
    double nd = 0., nn = 0.;
    {
      int const lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
      for(uint32_t i = r0 + w; i < r1; i += nw) {
        for(uint32_t c = (uint32_t) lane; c < R; c += 32) {
          double const x = (double) A(m)[(size_t) i * R + c], y = (double) Ao(m)[(size_t) i * R + c];
          nd = fma(y - x, y - x, nd);
          nn = fma(x, x, nn);
        }
      }
    }
    nd = warp_sum(nd);
    nn = warp_sum(nn);
    double * s = sm + sm_small(R) + 256;
    if(threadIdx.x < 2) { s[threadIdx.x] = 0.; }
    __syncthreads();
    if((threadIdx.x & 31) == 0) { atomicAdd(&s[0], nd); atomicAdd(&s[1], nn); }
    __syncthreads();
    if(threadIdx.x < 2) { atomicAdd(dacc(outer, mq) + threadIdx.x, s[threadIdx.x]); }
    zero_M(next_rows);
  }

  /* delta of an outer iteration: sum_m ||Aold - Anew|| / ||Anew|| */
  __device__ double delta(int outer) const
  {
    double d = 0.;
    for(int q = 0; q < a.nns; ++q) {
      d += sqrt(ldcg(dacc(outer, q) + 0)) / sqrt(ldcg(dacc(outer, q) + 1));
    }
    return d;
  }

  /* end of slice: forgetting, old <- new, time row out */
  __device__ void epilogue(int outer_its)
  {
    uint32_t const R = a.R;
    if(vb == 0) {
      double * Gt = a.G[a.sm];
      for(uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) { Gt[e] *= a.forget; }
      for(uint32_t c = threadIdx.x; c < R; c += blockDim.x) {
        if(a.time_out) { a.time_out[c] = a.s[c]; }
      }
      if(threadIdx.x == 0) { a.status[2] = outer_its; }
    }
    int const lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for(int q = 0; q < a.nns; ++q) {
      int const m = a.ns[q];
      uint32_t r0, r1;
      row_range(a.rows[m], vb, nvb, r0, r1);
      for(uint32_t i = r0 + w; i < r1; i += nw) {
        for(uint32_t c = (uint32_t) lane; c < R; c += 32) {
          Ao(m)[(size_t) i * R + c] = A(m)[(size_t) i * R + c];
        }
      }
    }
  }
};

/* dynamic shared memory needed by the phases for rank R */
static size_t stream_smem(uint32_t R)
{
  size_t a = (size_t) sm_xs(R) + (size_t) (ST_THREADS / 32) * 4 * SB_XS_STRIDE;
  size_t b = (size_t) 64 * R;
  return (a > b ? a : b) * sizeof(double);
}

/* ---- PLAIN executor: one phase per launch ---- */
template <typename T>
__global__ void __launch_bounds__(ST_THREADS, 1)
k_stream_phase(StreamArgs const a, int phase, int mq, int flag, uint32_t extra, int k)
{
  extern __shared__ double sm[];
  Ph<T> p{a, blockIdx.x, gridDim.x, sm};
  uint32_t const R = a.R;
  double * Ginv = sm + R * R;
  double * hb = sm + 2 * R * R;
  switch(phase) {
  case PH_NORM_PARTIAL: p.colnorm_partial(mq); break;
  case PH_NORM_APPLY: p.colnorm_apply(mq); break;
  case PH_GRAM: p.gram(mq); break;
  case PH_TIME_MTTKRP: p.time_mttkrp(extra); break;
  case PH_TIME_SOLVE: p.time_solve(); break;
  case PH_MODE_MTTKRP: p.mode_mttkrp_hist(mq, flag); break;
  case PH_ADMM_FIRST:
    if(flag) {
      p.mode_setup(mq, Ginv, hb);
      p.admm_first(mq, true, k, Ginv, hb, sm[sm_small(R) + 500]);
    } else {
      for(uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) { Ginv[e] = ldcg(a.Ginv + e); }
      __syncthreads();
      p.admm_first(mq, false, k, Ginv, hb, ldcg(a.red + RD_RHO));
    }
    break;
  case PH_ADMM_SECOND: p.admm_second(mq, k); break;
  case PH_MODE_FINISH: p.mode_finish(mq, flag, extra); break;
  case PH_EPILOGUE: p.epilogue(flag); break;
  default: break;
  }
}

/* ---- FUSED executor: one slice of one stream on a group of `nvb` blocks
 * (the whole grid for a single stream, a slice of it in a batch); phases are
 * separated by the stream's own bounded group barrier ---- */
template <typename T>
__device__ void run_slice(StreamArgs const & a, unsigned vb, unsigned nvb, double * sm)
{
  Ph<T> p{a, vb, nvb, sm};
  uint32_t const R = a.R;
  double * Ginv = sm + R * R;
  double * hb = sm + 2 * R * R;
#define SB_BAR() do { if(!grid_barrier(a.bar, a.status, nvb)) { return; } } while(0)

  p.clear_accumulators();
  SB_BAR();
  /* prologue (grow_mats): Grams of the grown factors, then on the first
   * slice the column normalisation (after the Gram, as the reference does) */
  for(int q = 0; q < a.nns; ++q) { p.gram(q); }
  SB_BAR();
  if(a.first_slice) {
    for(int q = 0; q < a.nns; ++q) { p.colnorm_partial(q); }
    SB_BAR();
    for(int q = 0; q < a.nns; ++q) { p.colnorm_apply(q); }
    SB_BAR();
  }

  double prev = 0.;
  int outer = 0;
  int inner_total = 0;
  int k = 0;                 /* ADMM phase counter (accumulator parity) */
  for(outer = 0; outer < a.max_outer; ++outer) {
    p.time_mttkrp(a.rows[a.ns[0]]);
    SB_BAR();
    p.time_solve();
    SB_BAR();
    for(int q = 0; q < a.nns; ++q) {
      p.mode_mttkrp_hist(q, outer);
      SB_BAR();
      p.mode_setup(q, Ginv, hb);
      double const rho = sm[sm_small(R) + 500];
      p.admm_first(q, true, k, Ginv, hb, rho);
      SB_BAR();
      /* One grid barrier per ADMM iteration: the second half of iteration
       * k and (speculatively) the first half of k+1 touch only this block's
       * rows; when the test after the barrier says k converged, P is
       * restored from init and the speculative accumulators are skipped. */
      int it = 0;
      while(true) {
        bool const last = (it + 1 >= a.max_inner);
        p.admm_step(q, k, !last, Ginv, rho);
        SB_BAR();
        bool const conv = p.admm_converged(k);
        ++it;
        if(conv || last) {
          if(!last) { p.admm_rollback(q); k += 2; } else { k += 1; }
          break;
        }
        k += 1;
      }
      inner_total += it;
      if(vb == 0 && threadIdx.x == 0) {
        a.status[4 + q] = it + (outer > 0 ? a.status[4 + q] : 0);
      }
      uint32_t const next_rows = (q + 1 < a.nns) ? a.rows[a.ns[q + 1]] : 0u;
      p.mode_finish(q, outer, next_rows);
      SB_BAR();
    }
    double const delta = p.delta(outer);
    if(outer > 0 && fabs(delta - prev) < a.outer_tol) { ++outer; break; }
    prev = delta;
  }
  if(outer > a.max_outer) { outer = a.max_outer; }
  p.epilogue(outer);
  if(vb == 0 && threadIdx.x == 0) { a.status[3] = inner_total; }
#undef SB_BAR
}

template <typename T>
__global__ void __launch_bounds__(ST_THREADS, 1)
k_stream_fused(StreamArgs const a)
{
  extern __shared__ double sm[];
  run_slice<T>(a, blockIdx.x, gridDim.x, sm);
}

/* ---- BATCHED executor: one slice from each of S independent streams in one
 * cooperative launch.  When S <= gridDim, stream s owns blocks
 * [grp[s], grp[s+1]) (sized by the host from its work); otherwise every
 * stream runs on a single block and block b takes streams b, b + gridDim, ...
 * in turn. ---- */
template <typename T>
__global__ void __launch_bounds__(ST_THREADS, 1)
k_stream_batched(StreamArgs const * __restrict__ args, int const * __restrict__ grp)
{
  int const S = __ldg(grp);                   /* grp[0] = S, offsets in grp[1..S+1] */
  grp += 1;
  extern __shared__ double sm[];
  __shared__ StreamArgs s_args;               /* this block's stream, in SMEM */
  auto load_args = [&](int s) {
    __syncthreads();
    static_assert(sizeof(StreamArgs) % 4 == 0, "StreamArgs copied as words");
    uint32_t const * src = (uint32_t const *) (args + s);
    uint32_t * dst = (uint32_t *) &s_args;
    for(uint32_t i = threadIdx.x; i < sizeof(StreamArgs) / 4; i += blockDim.x) { dst[i] = src[i]; }
    __syncthreads();
  };
  if(S <= (int) gridDim.x) {
    int lo = 0, hi = S;                       /* grp[lo] <= blockIdx.x < grp[hi] */
    while(hi - lo > 1) {
      int const mid = (lo + hi) >> 1;
      if(__ldg(grp + mid) <= (int) blockIdx.x) { lo = mid; } else { hi = mid; }
    }
    int const b0 = __ldg(grp + lo), b1 = __ldg(grp + lo + 1);
    if((int) blockIdx.x >= b1) { return; }   /* spare blocks */
    load_args(lo);
    run_slice<T>(s_args, blockIdx.x - b0, (unsigned) (b1 - b0), sm);
  } else {
    for(int s = blockIdx.x; s < S; s += gridDim.x) {
      load_args(s);
      run_slice<T>(s_args, 0u, 1u, sm);
    }
  }
}

/* per-slice error^2 of the latest slice, src/cpd/cpd.c:580-656 with lambda = 1:
 * MTTKRP over the time mode (in Mt), <X,Z> = s . Mt, ||Z||^2 = s^T
 * (Hadamard of the non-streamed Grams) s, all FP64 */
__global__ void k_local_err(StreamArgs const a, double xn, double * out)
{
  __shared__ double red[2];
  uint32_t const R = a.R;
  if(threadIdx.x < 2) { red[threadIdx.x] = 0.; }
  __syncthreads();
  double inner = 0., zn = 0.;
  for(uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) {
    uint32_t const i = e / R, j = e % R;
    double g = a.s[i] * a.s[j];
    for(int q = 0; q < a.nns; ++q) { g *= a.G[a.ns[q]][e]; }
    zn += g;
  }
  for(uint32_t c = threadIdx.x; c < R; c += blockDim.x) { inner += a.s[c] * a.Mt[c]; }
  atomicAdd(&red[0], inner);
  atomicAdd(&red[1], zn);
  __syncthreads();
  if(threadIdx.x == 0) { *out = (xn + fabs(red[1]) - 2. * red[0]) / xn; }
}

} /* namespace sb */

using namespace sb;

extern "C" {

int sb_stream_local_err(StreamArgs const * a, int vt, int nblocks, double xnormsq, double * out)
{
  SB_TRY(cudaMemsetAsync(a->Mt, 0, a->R * sizeof(double), stream()));
  int rc = sb_stream_phase(a, vt, PH_TIME_MTTKRP, 0, 0, 0u, 0, nblocks);
  if(rc) { return rc; }
  k_local_err<<<1, 256, 0, stream()>>>(*a, xnormsq, out);
  SB_CHECK_LAUNCH();
  return SB_OK;
}

size_t sb_stream_smem(uint32_t R) { return stream_smem(R); }
int sb_stream_threads(void) { return ST_THREADS; }

int sb_stream_blocks(uint32_t R, int vt)
{
  size_t const smem = stream_smem(R);
  int nb = 0, dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if(vt == SB_F64) {
    cudaFuncSetAttribute(k_stream_fused<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_stream_fused<double>, ST_THREADS, smem);
  } else {
    cudaFuncSetAttribute(k_stream_fused<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_stream_fused<float>, ST_THREADS, smem);
  }
  cudaGetLastError();
  if(nb < 1) { nb = 1; }
  return nb * nsm;
}

int sb_stream_phase(StreamArgs const * a, int vt, int phase, int mq, int flag, uint32_t extra,
    int k, int nblocks)
{
  size_t const smem = stream_smem(a->R);
  if(vt == SB_F64) {
    cudaFuncSetAttribute(k_stream_phase<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    k_stream_phase<double><<<nblocks, ST_THREADS, smem, stream()>>>(*a, phase, mq, flag, extra, k);
  } else {
    cudaFuncSetAttribute(k_stream_phase<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    k_stream_phase<float><<<nblocks, ST_THREADS, smem, stream()>>>(*a, phase, mq, flag, extra, k);
  }
  SB_CHECK_LAUNCH();
  return SB_OK;
}

int sb_stream_fused(StreamArgs const * a, int vt, int nblocks)
{
  size_t const smem = stream_smem(a->R);
  cudaLaunchConfig_t cfg;
  memset(&cfg, 0, sizeof(cfg));
  cfg.gridDim = dim3((unsigned) nblocks);
  cfg.blockDim = dim3(ST_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream();
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if(vt == SB_F64) {
    cudaFuncSetAttribute(k_stream_fused<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    SB_TRY(cudaLaunchKernelEx(&cfg, k_stream_fused<double>, *a));
  } else {
    cudaFuncSetAttribute(k_stream_fused<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    SB_TRY(cudaLaunchKernelEx(&cfg, k_stream_fused<float>, *a));
  }
  return SB_OK;
}

int sb_stream_batched(StreamArgs const * dargs, int const * dgrp, int vt, int nblocks,
    uint32_t Rmax)
{
  size_t const smem = stream_smem(Rmax);
  cudaLaunchConfig_t cfg;
  memset(&cfg, 0, sizeof(cfg));
  cfg.gridDim = dim3((unsigned) nblocks);
  cfg.blockDim = dim3(ST_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream();
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if(vt == SB_F64) {
    cudaFuncSetAttribute(k_stream_batched<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    SB_TRY(cudaLaunchKernelEx(&cfg, k_stream_batched<double>, dargs, dgrp));
  } else {
    cudaFuncSetAttribute(k_stream_batched<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    SB_TRY(cudaLaunchKernelEx(&cfg, k_stream_batched<float>, dargs, dgrp));
  }
  return SB_OK;
}

int sb_graph_capture_batch(void ** graph_exec, void * dst, void const * src_pinned, size_t bytes,
    StreamArgs const * dargs, int const * dgrp, int vt, int nblocks, uint32_t Rmax)
{
  *graph_exec = nullptr;
  cudaGraph_t g = nullptr;
  cudaStream_t const st = stream();
  SB_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaMemcpyAsync(dst, src_pinned, bytes, cudaMemcpyHostToDevice, st);
  int rc = (e == cudaSuccess) ? sb_stream_batched(dargs, dgrp, vt, nblocks, Rmax) : SB_EDEVICE;
  cudaError_t const e2 = cudaStreamEndCapture(st, &g);
  if(rc != SB_OK || e != cudaSuccess || e2 != cudaSuccess || g == nullptr) {
    if(g) { cudaGraphDestroy(g); }
    cudaGetLastError();
    return SB_EDEVICE;
  }
  cudaGraphExec_t ge = nullptr;
  e = cudaGraphInstantiate(&ge, g, 0);
  cudaGraphDestroy(g);
  if(e != cudaSuccess) { return fail(e); }
  *graph_exec = (void *) ge;
  return SB_OK;
}

} /* extern "C" */
