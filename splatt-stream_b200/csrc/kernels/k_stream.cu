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

/* threads per block: the single-stream kernels (fused, plain phases) run
 * 384, the scheduled multi-stream kernel 512 (its groups are small and the
 * rows per block many, where more warps hide more latency); shared-memory
 * staging is laid out for the larger, per-thread slots for the smaller */
constexpr int ST_THREADS_FUSED = 384;
constexpr int ST_THREADS_SCHED = 512;
constexpr int ST_THREADS_MAX = 512;
constexpr int ST_THREADS_MIN = 384;

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
  RD_CHUNK = RD_NACC + 512,   /* 8: chunked ADMM, sum of iterations x rows per mode */
  RD_SIMP = RD_CHUNK + 8,     /* 4 x 128: column simplex rounds (ring): 64 sums, 64 counts */
  RD_SIZE = RD_SIMP + SB_SIMP_RING * 128
};
static_assert(RD_NRM == SB_RD_NRM && RD_DACC == SB_RD_DACC && RD_CHUNK == SB_RD_CHUNK &&
              RD_SIMP == SB_RD_SIMP &&
              RD_SIZE <= SB_RED_SIZE,
    "red[] layout shared with the host");

template <typename T>
__device__ __forceinline__ T ldcg(T const * p) { return __ldcg(p); }

__device__ __forceinline__ unsigned long long gtimer()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

/* column simplex: threshold rounds per ADMM iteration at most (Michelot's
 * iteration settles in a handful; the bound only caps a pathological case) */
#define SB_SIMP_MAX_ROUNDS 64

/* deadline of every grid-barrier wait, in ns of %globaltimer (2 s unless
 * sb_set_wait_deadline_ns changed it: the failure-path tests shorten it so
 * that a wait that can never complete gives up within microseconds) */
__device__ unsigned long long g_wait_deadline_ns = 2000000000ull;

/* bounded grid barrier: returns false (in every thread) when the error flag
 * is set or the wait exceeded the deadline.  One word per barrier: arrival
 * count in the low 16 bits, generation in the high 16.  An arrival's
 * atomicAdd returns both; the last arrival resets the count and advances
 * the generation with one more add of 65536 - nblocks; the others poll the
 * word until its generation changes. */
__device__ bool grid_barrier(unsigned * bar, int * err, unsigned nblocks)
{
  __shared__ int s_ok;
  if(nblocks == 1) {           /* a group of one block: a block barrier */
    __threadfence();
    __syncthreads();
    return true;
  }
  __syncthreads();
  if(threadIdx.x == 0) {
    __threadfence();
    unsigned const old = atomicAdd(bar, 1u);
    unsigned const gen = old >> 16;
    int ok = 1;
    if((old & 0xffffu) == nblocks - 1) {
      atomicAdd(bar, 65536u - nblocks);
    } else {
      unsigned long long const t0 = gtimer();
      unsigned it = 0;
      while((*(volatile unsigned *) bar >> 16) == gen) {   /* error word and deadline every 64 polls */
        if((++it & 63u) == 0) {
          if(*(volatile int *) err) { ok = 0; break; }
          if(gtimer() - t0 > g_wait_deadline_ns) {
            atomicExch(err, 2);
            ok = 0;
            break;
          }
        }
      }
    }
    __threadfence();
    s_ok = ok;
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
  /* R <= 64 and blockDim >= ST_THREADS_MIN: at most NP (i, j) pairs per thread */
  constexpr int NP = (64 * 64 + ST_THREADS_MIN - 1) / ST_THREADS_MIN;
  double acc[NP];
#pragma unroll
  for(int q = 0; q < NP; ++q) { acc[q] = 0.; }
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
    for(int q = 0; q < NP; ++q) {
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
    for(int q = 0; q < NP; ++q) {
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

/* In-block FP64 Cholesky of S (R x R symmetric in shared memory, lower
 * triangle used; dpotrf('L') as mat_cholesky calls it,
 * src/matrix.c:104-124) and, when X is given, X = L^{-1} by forward
 * substitution in the same steps.  Returns the first bad pivot + 1 (0 if
 * positive definite; a bad pivot is replaced by 1 so the factorisation
 * completes).  Step k has two block barriers: (a) every thread takes
 * piv_k = sqrt(S[k][k]); threads k < t < R scale their column-k entry once
 * (l_t = S[t][k] / piv_k, into S and the column buffer col) and threads
 * t <= k divide X's row k by piv_k; (b) warps take the rows i > k and lanes
 * the columns: S[i][j] -= l_i l_j (k < j <= i) and X[i][c] -= l_i X[k][c]
 * (c <= k).  Every element gets the operations of the right-looking
 * factorisation and of the forward substitution in the same order as a
 * sequential loop would apply them; there is one division per row and step,
 * not per element, and no integer division.  col: R doubles of scratch. */
__device__ int block_chol(double * S, uint32_t R, double * X, double * col)
{
  __shared__ int s_bad;
  if(X) {
    for(uint32_t i = 0; i < R; ++i) {
      for(uint32_t c = threadIdx.x; c < R; c += blockDim.x) { X[i * R + c] = (i == c) ? 1. : 0.; }
    }
  }
  if(threadIdx.x == 0) { s_bad = 0; }
  __syncthreads();
  if(R <= 32 && blockDim.x >= 2 * R && R * R <= 3 * blockDim.x) {
    /* R <= 32: threads below R scale the column, threads R..2R-1 divide X's
     * row k (both need the pivot; no other thread computes it), and every
     * thread owns up to three fixed cells (i, j) of the R x R grid for the
     * updates: S[i][j] for k < j <= i, X[i][j] for j <= k < i (disjoint). */
    uint32_t ci[3], cj[3];
#pragma unroll
    for(int m = 0; m < 3; ++m) {
      uint32_t const e = threadIdx.x + (uint32_t) m * blockDim.x;
      ci[m] = e < R * R ? e / R : 0u;
      cj[m] = e < R * R ? e % R : 0u;
    }
    uint32_t const t = threadIdx.x;
    for(uint32_t k = 0; k < R; ++k) {
      double d = 0., piv = 1.;
      if(t < 2 * R) {
        d = S[k * R + k];
        piv = sqrt(d > 0. ? d : 1.);
        if(t < R) {
          if(t > k) {
            double const l = S[t * R + k] / piv;
            S[t * R + k] = l;
            col[t] = l;
          }
        } else if(X && t - R <= k) {
          X[k * R + (t - R)] /= piv;
        }
      }
      __syncthreads();
      if(t == 0) {
        S[k * R + k] = piv;
        if(!(d > 0.) && s_bad == 0) { s_bad = (int) k + 1; }
      }
#pragma unroll
      for(int m = 0; m < 3; ++m) {
        uint32_t const i = ci[m], j = cj[m];
        if(i > k) {
          if(j <= k) {
            if(X) { X[i * R + j] -= col[i] * X[k * R + j]; }
          } else if(j <= i) {
            S[i * R + j] -= col[i] * col[j];
          }
        }
      }
      __syncthreads();
    }
    return s_bad;
  }
  uint32_t const lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for(uint32_t k = 0; k < R; ++k) {
    double const d = S[k * R + k];
    double const piv = sqrt(d > 0. ? d : 1.);
    for(uint32_t t = threadIdx.x; t < R; t += blockDim.x) {
      if(t > k) {
        double const l = S[t * R + k] / piv;
        S[t * R + k] = l;
        col[t] = l;
      } else if(X) {
        X[k * R + t] /= piv;
      }
    }
    __syncthreads();
    if(threadIdx.x == 0) {
      S[k * R + k] = piv;
      if(!(d > 0.) && s_bad == 0) { s_bad = (int) k + 1; }
    }
    for(uint32_t i = k + 1 + w; i < R; i += nw) {
      double const li = col[i];
      for(uint32_t j = k + 1 + lane; j <= i; j += 32) { S[i * R + j] -= li * col[j]; }
      if(X) {
        for(uint32_t c = lane; c <= k; c += 32) { X[i * R + c] -= li * X[k * R + c]; }
      }
    }
    __syncthreads();
  }
  return s_bad;
}

/* Ginv = X^T X for X = L^{-1} (lower triangular, R x R in shared memory):
 * the inverse of L L^T */
__device__ void gram_of_inverse(double const * X, uint32_t R, double * Ginv)
{
  for(uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) {
    uint32_t const i = e / R, j = e % R;
    uint32_t const k0 = i > j ? i : j;
    double acc = 0.;
    for(uint32_t k = k0; k < R; ++k) { acc = fma(X[k * R + i], X[k * R + j], acc); }
    Ginv[e] = acc;
  }
  __syncthreads();
}

/* b <- (L L^T)^{-1} b for one vector (dpotrs), run by warp 0 alone with
 * __syncwarp between the substitution steps (a block barrier per step costs
 * more than the step); the same operations in the same order per element as
 * a block-wide substitution.  The whole block calls it; one block barrier at
 * the end. */
__device__ void warp_chol_solve_vec(double const * S, uint32_t R, double * b)
{
  if(threadIdx.x < 32) {
    uint32_t const lane = threadIdx.x;
    for(uint32_t i = 0; i < R; ++i) {
      if(lane == 0) { b[i] /= S[i * R + i]; }
      __syncwarp();
      double const yi = b[i];
      for(uint32_t k = i + 1 + lane; k < R; k += 32) { b[k] -= S[k * R + i] * yi; }
      __syncwarp();
    }
    for(uint32_t ii = R; ii-- > 0; ) {
      if(lane == 0) { b[ii] /= S[ii * R + ii]; }
      __syncwarp();
      double const xi = b[ii];
      for(uint32_t k = lane; k < ii; k += 32) { b[k] -= S[ii * R + k] * xi; }
      __syncwarp();
    }
  }
  __syncthreads();
}

/* ------------------------------------------------------------------------ */
/* phases                                                                    */
/* ------------------------------------------------------------------------ */
/* The prox of one primal element (maxcolnorm.c:32-62,
 * maxcolnorm-nonneg.c:32-62): cn / rcn are the column's 2-norm and its
 * reciprocal.  A scaled result is rounded to the stored type as the primal
 * is. */
template <typename T>
__device__ __forceinline__ double prox_apply(int kind, double p, double cn, double rcn)
{
  if(kind == SB_PROX_MAXCOLNORM_NONNEG && !(p > 0.)) { return 0.; }
  return cn > 1. ? (double) (T) (p * rcn) : p;
}

/* the pre-prox primal as it enters its column's squared norm: the
 * non-negative kind measures the column after zeroing its negatives */
__device__ __forceinline__ double prox_norm_elem(int kind, double np)
{
  return (kind == SB_PROX_MAXCOLNORM_NONNEG && !(np > 0.)) ? 0. : np;
}

/* NN: whether a mode may carry the non-negative prox (false compiles the
 * max-column-norm row passes only) */
template <typename T, bool NN = true>
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
    /* a Gram that is carried over (rows0 > 0) already holds the product of
     * its factor's old rows: the last mode update of the previous slice
     * left G = A^T A of the factor as it stands */
    for(int q = 0; q < a.nns; ++q) {
      if(a.rows0[a.ns[q]] > 0) { continue; }
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
  /* G[m] += A^T A over the factor's rows [from, rows): all rows (the
   * PLAIN executor, which clears G first), or only the rows this slice added
   * (the fused executors, whose G carries the old rows' product over) */
  __device__ void gram(int q, bool grown_only)
  {
    int const m = a.ns[q];
    uint32_t const from = grown_only ? a.rows0[m] : 0u;
    uint32_t r0, r1;
    row_range(a.rows[m] - from, vb, nvb, r0, r1);
    block_cross_add<T>(A(m), A(m), from + r0, from + r1, a.R, a.G[m], sm);
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
      bool const okc = c < R;
      double acc = 0.;          /* FP64 products and sums for either value type */
      /* eight nonzeros per step: their index loads, then their row gathers,
       * are issued together (the phase is bound by the gathers' latency) */
      for(uint32_t n = n0 + 8 * w; n < n1; n += 8 * nw) {
        uint32_t const cnt = umin32(8, n1 - n);
        double p[8];
#pragma unroll
        for(int j = 0; j < 8; ++j) { p[j] = ((uint32_t) j < cnt) ? (double) __ldg(vals + n + j) : 0.; }
        for(int q = 0; q < a.nns; ++q) {
          T const * Am = A(a.ns[q]);
          uint32_t const * im = a.inds[a.ns[q]];
          uint32_t id[8];
#pragma unroll
          for(int j = 0; j < 8; ++j) { id[j] = ((uint32_t) j < cnt) ? __ldg(im + n + j) : 0u; }
#pragma unroll
          for(int j = 0; j < 8; ++j) {
            p[j] *= ((uint32_t) j < cnt && okc) ? (double) ldcg(Am + (size_t) id[j] * R + c) : 0.;
          }
        }
        acc += ((p[0] + p[1]) + (p[2] + p[3])) + ((p[4] + p[5]) + (p[6] + p[7]));
      }
      v[h] = acc;
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
    int bad = block_chol(S, R, nullptr, sm + sm_big(R) + R * R);
    if(threadIdx.x == 0 && bad) { atomicMax(a.status + 1, bad); }
    double * y = sm + sm_small(R);
    for(uint32_t c = threadIdx.x; c < R; c += blockDim.x) { y[c] = ldcg(a.Mt + c); }
    __syncthreads();
    warp_chol_solve_vec(S, R, y);
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
    /* FP64: output rows below `hot` gather their partial sums in shared
     * memory (the first 3 R^2 doubles are free in this phase) and reach M
     * with one atomic per element per block at the end.  Under the
     * first-appearance relabelling the most frequent rows of a skewed stream
     * get the lowest ids; their FP64 global atomics would otherwise
     * serialise on a few addresses (measured: 59 -> 36 us for the c2 stream's
     * second mode).  FP32 global atomics keep up, and the staging only costs
     * there. */
    T * const hs = (T *) sm;
    uint32_t const hot = sizeof(T) == 8 ? umin32(a.rows[m], 3 * R) : 0u;
    for(uint32_t e = threadIdx.x; e < hot * R; e += blockDim.x) { hs[e] = (T) 0; }
    __syncthreads();
    for(uint32_t c0 = 0; c0 < R; c0 += 32) {
      uint32_t const c = c0 + lane;
      bool const okc = c < R;
      /* the time factor row (slice index 0) */
      double const st = okc ? (double) ldcg((T const *) a.sT + c) : 0.;
      double acc = 0.;          /* FP64 products and run sums for either value type */
      uint32_t run = 0xffffffffu;
      /* eight nonzeros per step: output indices, values, the other modes'
       * indices and row gathers are issued together (the phase is bound by
       * the gathers' latency); the run of equal output rows is then followed
       * in order */
      for(uint32_t n = w0; n < w1; n += 8) {
        uint32_t const cnt = umin32(8, w1 - n);
        uint32_t o[8];
        double p[8];
#pragma unroll
        for(int j = 0; j < 8; ++j) {
          bool const v = (uint32_t) j < cnt;
          o[j] = v ? __ldg(oind + n + j) : 0xffffffffu;
          p[j] = v ? (double) __ldg(vals + n + j) : 0.;
        }
        for(int q = 0; q < a.nns; ++q) {
          int const k = a.ns[q];
          if(k == m) { continue; }
          T const * Ak = A(k);
          uint32_t const * ik = a.inds[k];
          uint32_t id[8];
#pragma unroll
          for(int j = 0; j < 8; ++j) { id[j] = ((uint32_t) j < cnt) ? __ldg(ik + n + j) : 0u; }
#pragma unroll
          for(int j = 0; j < 8; ++j) {
            p[j] *= ((uint32_t) j < cnt && okc) ? (double) ldcg(Ak + (size_t) id[j] * R + c) : 0.;
          }
        }
#pragma unroll
        for(int j = 0; j < 8; ++j) {
          if((uint32_t) j >= cnt) { break; }
          if(o[j] != run) {
            if(run != 0xffffffffu && okc) {
              atomicAdd((run < hot ? hs : M()) + (size_t) run * R + c, (T) acc);
            }
            acc = 0.;
            run = o[j];
          }
          acc += p[j] * st;   /* the product order of the per-nonzero loop */
        }
      }
      if(run != 0xffffffffu && okc) {
        atomicAdd((run < hot ? hs : M()) + (size_t) run * R + c, (T) acc);
      }
    }
    __syncthreads();
    for(uint32_t e = threadIdx.x; e < hot * R; e += blockDim.x) {
      T const v = hs[e];
      if(v != (T) 0) { atomicAdd(M() + e, v); }
    }
    __syncthreads();
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
    int const bad = block_chol(S, R, sm + sm_big(R), sm + sm_big(R) + R * R);
    if(threadIdx.x == 0 && bad && vb == 0) { atomicMax(a.status + 1, bad); }
    gram_of_inverse(sm + sm_big(R), R, Ginv);
    if(vb == 0) {
      for(uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) { a.Ginv[e] = Ginv[e]; }
      if(threadIdx.x == 0) { a.red[RD_RHO] = s_rho; }
    }
    sm[sm_small(R) + 500] = s_rho;   /* block-local copy for admm_first */
    __syncthreads();
  }

  /* y[rr][h] = sum_q x[rr][q] * G[q][lane + 32 h] for the warp's four rows
   * staged in xs (row stride SB_XS_STRIDE); G is R x R double in shared
   * memory.  One element of G serves four rows. */
  template <int H>
  __device__ __forceinline__ void prod4(T const * xs, double const * G, uint32_t R, int lane,
      double (&y)[4][H]) const
  {
#pragma unroll
    for(int rr = 0; rr < 4; ++rr) {
#pragma unroll
      for(int h = 0; h < H; ++h) { y[rr][h] = 0.; }
    }
    for(uint32_t q = 0; q < R; q += 2) {
      bool const two = q + 1 < R;
      double g0[H], g1[H];
#pragma unroll
      for(int h = 0; h < H; ++h) {
        uint32_t const c = (uint32_t) lane + 32u * h;
        bool const ok = c < R;
        g0[h] = ok ? G[q * R + c] : 0.;
        g1[h] = (ok && two) ? G[(q + 1) * R + c] : 0.;
      }
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
#pragma unroll
        for(int h = 0; h < H; ++h) { y[rr][h] = fma(xa, g0[h], fma(xb, g1[h], y[rr][h])); }
      }
    }
  }

  /* FP32, R <= 32: the same product with G's column `lane` in registers */
  __device__ __forceinline__ void prod4_reg(float const * xf, float const (&gcol)[32], uint32_t R,
      double (&y)[4][1]) const
  {
#pragma unroll
    for(int rr = 0; rr < 4; ++rr) { y[rr][0] = 0.; }
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
        y[rr][0] += (double) acc;
      }
    }
  }

  template <int H>
  __device__ __forceinline__ void prod4_any(T const * xs, double const * G, float const (&gcol)[32],
      uint32_t R, int lane, double (&y)[4][H]) const
  {
    if constexpr (H == 1 && sizeof(T) == 4) {
      prod4_reg((float const *) xs, gcol, R, y);
    } else {
      prod4<H>(xs, G, R, lane, y);
    }
  }

  /* ADMM first half for this block's rows: (first: M += Aold hb, D = 0),
   * init = P, aux = (M + rho (P + D)) Ginv, P = aux - D, column sums of P^2
   * into cn_acc(k); block 0 clears cn_acc(k+1) (and G[m] on the first).
   * Warps take four rows at a time: all loads of the four rows are issued
   * before any store, the two row products run on the staged rows.
   * H = column halves per lane (1 for R <= 32, 2 up to 64). */
  template <int H, int PK>
  __device__ void admm_first_h(int mq, bool first, int k, double const * Ginv, double const * hb,
      double rho)
  {
    int const m = a.ns[mq];
    constexpr int pk = PK;
    uint32_t const R = a.R;
    if(vb == 0) {
      for(uint32_t c = threadIdx.x; c < 64; c += blockDim.x) { cn_acc(k + 1)[c] = 0.; }
      if(threadIdx.x < 4) { nrm_acc(k + 1)[threadIdx.x] = 0.; }
      if(a.prox[m] == SB_PROX_COLSIMP) {
        /* the column simplex's round 0 accumulates into slot 0 next */
        for(uint32_t c = threadIdx.x; c < 128; c += blockDim.x) { a.red[RD_SIMP + c] = 0.; }
      }
      if(first) {
        for(uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) { a.G[m][e] = 0.; }
      }
    }
    uint32_t r0, r1;
    row_range(a.rows[m], vb, nvb, r0, r1);
    int const lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    T * xs = (T *) (sm + sm_xs(R)) + (size_t) w * 4 * SB_XS_STRIDE;
    float gcol[32];
    if constexpr (H == 1 && sizeof(T) == 4) {
#pragma unroll
      for(int q = 0; q < 32; ++q) {
        gcol[q] = ((uint32_t) q < R && (uint32_t) lane < R) ? (float) Ginv[q * R + lane] : 0.f;
      }
    }
    double cs[H];
#pragma unroll
    for(int h = 0; h < H; ++h) { cs[h] = 0.; }
    T * __restrict__ P = A(m);
    T * __restrict__ D = Dm(m);
    T * __restrict__ Mb = M();
    T * __restrict__ IN = INIT();
    T * __restrict__ AU = AUX();
    T const * __restrict__ AO = Ao(m);
    for(uint32_t i0 = r0 + 4 * w; i0 < r1; i0 += 4 * nw) {
      uint32_t const nr = umin32(4, r1 - i0);
      T lm[4][H], lp[4][H], ld[4][H];
#pragma unroll
      for(int rr = 0; rr < 4; ++rr) {
#pragma unroll
        for(int h = 0; h < H; ++h) {
          uint32_t const c = (uint32_t) lane + 32u * h;
          bool const v = (uint32_t) rr < nr && c < R;
          size_t const b = (size_t) (i0 + rr) * R + c;
          /* M rows were accumulated by other blocks' atomics: read through L2 */
          lm[rr][h] = v ? ldcg(Mb + b) : (T) 0;
          lp[rr][h] = v ? P[b] : (T) 0;
          ld[rr][h] = v ? (first ? AO[b] : D[b]) : (T) 0;
        }
      }
      double mm[4][H], dd[4][H];
      if(first) {
        /* M += Aold[i] * hb  (add_historical, StreamCPD.cc:274-291) */
#pragma unroll
        for(int rr = 0; rr < 4; ++rr) {
#pragma unroll
          for(int h = 0; h < H; ++h) {
            uint32_t const c = (uint32_t) lane + 32u * h;
            if(c < R) { xs[rr * SB_XS_STRIDE + c] = ld[rr][h]; }
          }
        }
        __syncwarp();
        double yh[4][H];
        prod4<H>(xs, hb, R, lane, yh);
        __syncwarp();
#pragma unroll
        for(int rr = 0; rr < 4; ++rr) {
#pragma unroll
          for(int h = 0; h < H; ++h) {
            uint32_t const c = (uint32_t) lane + 32u * h;
            mm[rr][h] = (double) (T) ((double) lm[rr][h] + yh[rr][h]);
            dd[rr][h] = 0.;
            if((uint32_t) rr < nr && c < R) {
              size_t const b = (size_t) (i0 + rr) * R + c;
              Mb[b] = (T) mm[rr][h];
              D[b] = (T) 0;
            }
          }
        }
      } else {
#pragma unroll
        for(int rr = 0; rr < 4; ++rr) {
#pragma unroll
          for(int h = 0; h < H; ++h) { mm[rr][h] = (double) lm[rr][h]; dd[rr][h] = (double) ld[rr][h]; }
        }
      }
#pragma unroll
      for(int rr = 0; rr < 4; ++rr) {
#pragma unroll
        for(int h = 0; h < H; ++h) {
          uint32_t const c = (uint32_t) lane + 32u * h;
          if(c >= R) { continue; }
          double const p = (double) lp[rr][h];
          if((uint32_t) rr < nr) { IN[(size_t) (i0 + rr) * R + c] = lp[rr][h]; }
          /* the reference's auxiliary: M + rho (P + D)  (src/cpd/admm.c:51) */
          xs[rr * SB_XS_STRIDE + c] = (T) (mm[rr][h] + rho * (p + dd[rr][h]));
        }
      }
      __syncwarp();
      double y[4][H];
      prod4_any<H>(xs, Ginv, gcol, R, lane, y);
      __syncwarp();
#pragma unroll
      for(int rr = 0; rr < 4; ++rr) {
#pragma unroll
        for(int h = 0; h < H; ++h) {
          uint32_t const c = (uint32_t) lane + 32u * h;
          if((uint32_t) rr >= nr || c >= R) { continue; }
          size_t const b = (size_t) (i0 + rr) * R + c;
          T const au = (T) y[rr][h];
          T const np = (T) ((double) au - dd[rr][h]);
          AU[b] = au;
          P[b] = np;
          double const q = prox_norm_elem(pk, (double) np);
          cs[h] = fma(q, q, cs[h]);
        }
      }
    }
    block_cols_add(sm + sm_small(R), R, (uint32_t) lane, cs[0], H > 1 ? cs[H - 1] : 0.,
        (uint32_t) lane < R, (uint32_t) lane + 32 < R, cn_acc(k));
  }

  __device__ void admm_first(int mq, bool first, int k, double const * Ginv, double const * hb,
      double rho)
  {
    /* the prox kind is uniform over the mode: one instantiation per kind */
    bool const nn = NN && a.prox[a.ns[mq]] == SB_PROX_MAXCOLNORM_NONNEG;
    if(a.R <= 32) {
      if(nn) { admm_first_h<1, SB_PROX_MAXCOLNORM_NONNEG>(mq, first, k, Ginv, hb, rho); }
      else { admm_first_h<1, SB_PROX_MAXCOLNORM>(mq, first, k, Ginv, hb, rho); }
    } else {
      if(nn) { admm_first_h<2, SB_PROX_MAXCOLNORM_NONNEG>(mq, first, k, Ginv, hb, rho); }
      else { admm_first_h<2, SB_PROX_MAXCOLNORM>(mq, first, k, Ginv, hb, rho); }
    }
  }

  /* ADMM second half: prox (columns with norm > 1 scaled to unit norm),
   * D += P - aux, the four norms into nrm_acc(k) */
  __device__ void admm_second(int mq, int k)
  {
    int const m = a.ns[mq];
    int const pk = a.prox[m];
    uint32_t const R = a.R;
    uint32_t r0, r1;
    row_range(a.rows[m], vb, nvb, r0, r1);
    double * cn = sm + sm_small(R) + 128;
    double * rcn = sm + sm_small(R) + 192;
    for(uint32_t c = threadIdx.x; c < R; c += blockDim.x) {
      cn[c] = sqrt(ldcg(cn_acc(k) + c));
      rcn[c] = cn[c] > 0. ? 1. / cn[c] : 0.;   /* as the fused step */
    }
    __syncthreads();
    double dn = 0., pn = 0., pr = 0., dr = 0.;
    T * P = A(m);
    T * D = Dm(m);
    for(uint64_t e = (uint64_t) r0 * R + threadIdx.x; e < (uint64_t) r1 * R; e += blockDim.x) {
      uint32_t const c = (uint32_t) (e % R);
      double p = (double) P[e];
      p = prox_apply<T>(pk, p, cn[c], rcn[c]);
      P[e] = (T) p;
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
   * Each warp takes four rows at a time: every load of the four rows is
   * issued before any store (restrict-qualified), the new duals stay in
   * registers for the first half, and the rows' auxiliary inputs x are
   * staged in the warp's shared-memory slice for the row-times-
   * (G + rho I)^-1 product (one inverse element serves four rows; FP32 with
   * R <= 32 keeps the inverse's column in registers). */
  template <int H, int PK>
  __device__ void admm_step_h(int mq, int k, bool spec, double const * Ginv, double rho,
      bool cn_staged)
  {
    int const m = a.ns[mq];
    constexpr int pk = PK;
    uint32_t const R = a.R;
    if(spec && vb == 0) {
      for(uint32_t c = threadIdx.x; c < 64; c += blockDim.x) { cn_acc(k + 2)[c] = 0.; }
      if(threadIdx.x < 4) { nrm_acc(k + 2)[threadIdx.x] = 0.; }
    }
    double * cn = sm + sm_small(R) + 128;
    if(!cn_staged) {             /* else loaded with the previous convergence test */
      for(uint32_t c = threadIdx.x; c < R; c += blockDim.x) { cn[c] = sqrt(ldcg(cn_acc(k) + c)); }
      __syncthreads();
    }
    uint32_t r0, r1;
    row_range(a.rows[m], vb, nvb, r0, r1);
    int const lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double cnv[H];
#pragma unroll
    for(int h = 0; h < H; ++h) {
      uint32_t const c = (uint32_t) lane + 32u * h;
      cnv[h] = c < R ? cn[c] : 0.;
    }
    /* columns with norm > 1 are scaled by the norm's reciprocal (one
     * division per column instead of one per element) */
    double rcn[H];
#pragma unroll
    for(int h = 0; h < H; ++h) { rcn[h] = cnv[h] > 0. ? 1. / cnv[h] : 0.; }
    T * xs = (T *) (sm + sm_xs(R)) + (size_t) w * 4 * SB_XS_STRIDE;   /* this warp's 4 rows */
    float gcol[32];
    if constexpr (H == 1 && sizeof(T) == 4) {
#pragma unroll
      for(int q = 0; q < 32; ++q) {
        gcol[q] = ((uint32_t) q < R && (uint32_t) lane < R) ? (float) Ginv[q * R + lane] : 0.f;
      }
    }
    double dn = 0., pn = 0., pr = 0., dr = 0.;
    double cs[H];
#pragma unroll
    for(int h = 0; h < H; ++h) { cs[h] = 0.; }
    T * __restrict__ P = A(m);
    T * __restrict__ D = Dm(m);
    T * __restrict__ AU = AUX();
    T * __restrict__ IN = INIT();
    T const * __restrict__ Mb = M();
    for(uint32_t i0 = r0 + 4 * w; i0 < r1; i0 += 4 * nw) {
      uint32_t const nr = umin32(4, r1 - i0);
      T lp[4][H], lau[4][H], ld[4][H], lin[4][H], lm[4][H];
#pragma unroll
      for(int rr = 0; rr < 4; ++rr) {
#pragma unroll
        for(int h = 0; h < H; ++h) {
          uint32_t const c = (uint32_t) lane + 32u * h;
          bool const v = (uint32_t) rr < nr && c < R;
          size_t const b = (size_t) (i0 + rr) * R + c;
          lau[rr][h] = v ? AU[b] : (T) 0;
          ld[rr][h] = v ? D[b] : (T) 0;
          lin[rr][h] = v ? IN[b] : (T) 0;
          lm[rr][h] = (v && spec) ? ldcg(Mb + b) : (T) 0;
          /* the pre-prox primal is aux - D, exactly as the previous first
           * half rounded and stored it: not kept in memory during the loop */
          lp[rr][h] = (T) ((double) lau[rr][h] - (double) ld[rr][h]);
        }
      }
      /* second half of iteration k */
      double dk[4][H];
#pragma unroll
      for(int rr = 0; rr < 4; ++rr) {
#pragma unroll
        for(int h = 0; h < H; ++h) {
          uint32_t const c = (uint32_t) lane + 32u * h;
          dk[rr][h] = 0.;
          if((uint32_t) rr >= nr || c >= R) { continue; }
          size_t const b = (size_t) (i0 + rr) * R + c;
          double const p = prox_apply<T>(pk, (double) lp[rr][h], cnv[h], rcn[h]);
          double const au = (double) lau[rr][h];
          double const d = (double) (T) ((double) ld[rr][h] + p - au);
          double const pd = p - au, dd = p - (double) lin[rr][h];
          dn = fma(d, d, dn); pn = fma(p, p, pn); pr = fma(pd, pd, pr); dr = fma(dd, dd, dr);
          D[b] = (T) d;
          if(!spec) {
            P[b] = (T) p;
          } else {
            IN[b] = (T) p;
            dk[rr][h] = d;
            xs[rr * SB_XS_STRIDE + c] = (T) ((double) lm[rr][h] + rho * (p + d));
          }
        }
      }
      if(!spec) { continue; }
      __syncwarp();
      double y[4][H];
      prod4_any<H>(xs, Ginv, gcol, R, lane, y);
      __syncwarp();
      /* first half of iteration k+1: aux = y, P = aux - D */
#pragma unroll
      for(int rr = 0; rr < 4; ++rr) {
#pragma unroll
        for(int h = 0; h < H; ++h) {
          uint32_t const c = (uint32_t) lane + 32u * h;
          if((uint32_t) rr >= nr || c >= R) { continue; }
          size_t const b = (size_t) (i0 + rr) * R + c;
          T const au = (T) y[rr][h];
          T const np = (T) ((double) au - dk[rr][h]);   /* P, implicit: aux - D */
          AU[b] = au;
          double const q = prox_norm_elem(pk, (double) np);
          cs[h] = fma(q, q, cs[h]);
        }
      }
    }
    /* the four norms of iteration k and the column sums of the new primal
     * (lane c holds column c's): each warp leaves its partials in its own
     * staging slice (free now), one block barrier, then thread t sums
     * column t (t < R) or norm t - R across the warps and adds it to the
     * global accumulator */
    dn = warp_sum(dn); pn = warp_sum(pn); pr = warp_sum(pr); dr = warp_sum(dr);
    __syncwarp();
    /* warp w's partials live in its own staging slice (4 * SB_XS_STRIDE
     * values of T: 1 KB for FP32, room for R + 4 <= 68 doubles) */
    constexpr size_t slice = (size_t) 4 * SB_XS_STRIDE * sizeof(T);
    unsigned char * part = (unsigned char *) (sm + sm_xs(R));
    double * mine = (double *) (part + (size_t) w * slice);
    if(spec) {
#pragma unroll
      for(int h = 0; h < H; ++h) {
        uint32_t const c = (uint32_t) lane + 32u * h;
        if(c < R) { mine[c] = cs[h]; }
      }
    }
    if(lane == 0) { mine[R] = dn; mine[R + 1] = pn; mine[R + 2] = pr; mine[R + 3] = dr; }
    __syncthreads();
    uint32_t const t = threadIdx.x;
    if(t < R + 4 && (spec || t >= R)) {
      double acc = 0.;
      for(int ww = 0; ww < nw; ++ww) { acc += ((double const *) (part + (size_t) ww * slice))[t]; }
      if(t < R) { atomicAdd(cn_acc(k + 1) + t, acc); }
      else { atomicAdd(nrm_acc(k) + (t - R), acc); }
    }
  }

  __device__ void admm_step(int mq, int k, bool spec, double const * Ginv, double rho,
      bool cn_staged = false)
  {
    bool const nn = NN && a.prox[a.ns[mq]] == SB_PROX_MAXCOLNORM_NONNEG;
    if(a.R <= 32) {
      if(nn) { admm_step_h<1, SB_PROX_MAXCOLNORM_NONNEG>(mq, k, spec, Ginv, rho, cn_staged); }
      else { admm_step_h<1, SB_PROX_MAXCOLNORM>(mq, k, spec, Ginv, rho, cn_staged); }
    } else {
      if(nn) { admm_step_h<2, SB_PROX_MAXCOLNORM_NONNEG>(mq, k, spec, Ginv, rho, cn_staged); }
      else { admm_step_h<2, SB_PROX_MAXCOLNORM>(mq, k, spec, Ginv, rho, cn_staged); }
    }
  }

  /* Row-separable ADMM (lasso, lasso.c:32-55; the row simplex, simplex.cc:
   * 34-66; the NTF regularizations, nonneg_lasso.c:30-45 and
   * nonneg_frob.c:31-49) as the reference runs it for such constraints:
   * independent chunks of chunk[m] rows, each iterating until its own
   * residual test passes (src/cpd/admm.c:352-395, 240-308).
   * A warp owns whole chunks, so no block or grid synchronisation is needed:
   * per chunk it first adds the historical term and clears the duals (what
   * the first half does for the other proxes), then per iteration and row
   * group of four: aux = (M + rho (P + D)) (G + rho I)^-1, P = aux - D, the
   * prox, D += P - aux, and the chunk's four norms.  Iterations x rows per
   * chunk add into red[RD_CHUNK + mq]. */
  template <int H>
  __device__ void admm_chunked_h(int mq, double const * Ginv, double const * hb, double rho)
  {
    int const m = a.ns[mq];
    uint32_t const R = a.R;
    uint32_t const rows = a.rows[m];
    uint32_t const C = a.chunk[m] ? a.chunk[m] : 50u;
    int const pk = a.prox[m];
    double const thr = a.prox_mult[m] / rho;
    if(vb == 0) {
      for(uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) { a.G[m][e] = 0.; }
    }
    int const lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    T * xs = (T *) (sm + sm_xs(R)) + (size_t) w * 4 * SB_XS_STRIDE;
    float gcol[32];
    if constexpr (H == 1 && sizeof(T) == 4) {
#pragma unroll
      for(int q = 0; q < 32; ++q) {
        gcol[q] = ((uint32_t) q < R && (uint32_t) lane < R) ? (float) Ginv[q * R + lane] : 0.f;
      }
    }
    T * __restrict__ P = A(m);
    T * __restrict__ D = Dm(m);
    T * __restrict__ Mb = M();
    T const * __restrict__ AO = Ao(m);
    uint32_t const nchunks = (rows + C - 1) / C;
    for(uint32_t ch = vb * (uint32_t) nw + (uint32_t) w; ch < nchunks; ch += nvb * (uint32_t) nw) {
      uint32_t const c0 = ch * C, c1 = umin32(c0 + C, rows);
      /* M += Aold * hb (add_historical), D = 0 */
      for(uint32_t i0 = c0; i0 < c1; i0 += 4) {
        uint32_t const nr = umin32(4, c1 - i0);
#pragma unroll
        for(int rr = 0; rr < 4; ++rr) {
#pragma unroll
          for(int h = 0; h < H; ++h) {
            uint32_t const c = (uint32_t) lane + 32u * h;
            if(c < R) {
              xs[rr * SB_XS_STRIDE + c] =
                  (uint32_t) rr < nr ? AO[(size_t) (i0 + rr) * R + c] : (T) 0;
            }
          }
        }
        __syncwarp();
        double yh[4][H];
        prod4<H>(xs, hb, R, lane, yh);
        __syncwarp();
#pragma unroll
        for(int rr = 0; rr < 4; ++rr) {
#pragma unroll
          for(int h = 0; h < H; ++h) {
            uint32_t const c = (uint32_t) lane + 32u * h;
            if((uint32_t) rr >= nr || c >= R) { continue; }
            size_t const b = (size_t) (i0 + rr) * R + c;
            Mb[b] = (T) ((double) ldcg(Mb + b) + yh[rr][h]);
            D[b] = (T) 0;
          }
        }
      }
      __syncwarp();
      int it;
      for(it = 0; it < a.max_inner; ++it) {
        double dn = 0., pn = 0., pr = 0., dr = 0.;
        for(uint32_t i0 = c0; i0 < c1; i0 += 4) {
          uint32_t const nr = umin32(4, c1 - i0);
          double lp[4][H], ld[4][H];
#pragma unroll
          for(int rr = 0; rr < 4; ++rr) {
#pragma unroll
            for(int h = 0; h < H; ++h) {
              uint32_t const c = (uint32_t) lane + 32u * h;
              bool const v = (uint32_t) rr < nr && c < R;
              size_t const b = (size_t) (i0 + rr) * R + c;
              lp[rr][h] = v ? (double) P[b] : 0.;
              ld[rr][h] = v ? (double) D[b] : 0.;
              double const mm = v ? (double) Mb[b] : 0.;
              /* auxiliary: M + rho (P + D)  (src/cpd/admm.c:51) */
              if(c < R) { xs[rr * SB_XS_STRIDE + c] = (T) (mm + rho * (lp[rr][h] + ld[rr][h])); }
            }
          }
          __syncwarp();
          double y[4][H];
          prod4_any<H>(xs, Ginv, gcol, R, lane, y);
          __syncwarp();
          /* P = aux - D, then the row-separable prox */
          double pa[4][H], pp[4][H];
#pragma unroll
          for(int rr = 0; rr < 4; ++rr) {
#pragma unroll
            for(int h = 0; h < H; ++h) {
              pa[rr][h] = (double) (T) y[rr][h];
              pp[rr][h] = (double) (T) (pa[rr][h] - ld[rr][h]);
            }
          }
          if(pk == SB_PROX_ROWSIMP) {
            /* each row onto the probability simplex (simplex.cc:34-66):
             * lane rr sorts row rr and takes the reference's running-sum
             * pivot in the same order; theta then goes to every lane */
#pragma unroll
            for(int rr = 0; rr < 4; ++rr) {
#pragma unroll
              for(int h = 0; h < H; ++h) {
                uint32_t const c = (uint32_t) lane + 32u * h;
                if(c < R) { xs[rr * SB_XS_STRIDE + c] = (T) pp[rr][h]; }
              }
            }
            __syncwarp();
            double theta = 0.;
            if((uint32_t) lane < nr) {
              double buf[64];
              T const * row = xs + lane * SB_XS_STRIDE;
              for(uint32_t j = 0; j < R; ++j) {             /* insertion sort, descending */
                double const x = (double) row[j];
                uint32_t q = j;
                while(q > 0 && buf[q - 1] < x) { buf[q] = buf[q - 1]; --q; }
                buf[q] = x;
              }
              double run = -1.;
              uint32_t piv;
              for(piv = 0; piv < R; ++piv) {
                run += buf[piv];
                if(buf[piv] - run / (double) (piv + 1) <= 0.) { run -= buf[piv]; break; }
              }
              theta = run / (double) piv;
            }
            __syncwarp();
#pragma unroll
            for(int rr = 0; rr < 4; ++rr) {
              double const th = __shfl_sync(0xffffffffu, theta, rr);
#pragma unroll
              for(int h = 0; h < H; ++h) {
                double const x = pp[rr][h] - th;
                pp[rr][h] = (double) (T) (x > 0. ? x : 0.);
              }
            }
          } else if(pk == SB_PROX_NTF_LASSO) {
            /* one-sided threshold: the L1 prox on the non-negative orthant */
#pragma unroll
            for(int rr = 0; rr < 4; ++rr) {
#pragma unroll
              for(int h = 0; h < H; ++h) {
                double const x = pp[rr][h];
                pp[rr][h] = (double) (T) (x > thr ? x - thr : 0.);
              }
            }
          } else if(pk == SB_PROX_NTF_FROB) {
            /* the Frobenius shrink rho / (multiplier + rho), then negatives zeroed */
            double const shrink = rho / (a.prox_mult[m] + rho);
#pragma unroll
            for(int rr = 0; rr < 4; ++rr) {
#pragma unroll
              for(int h = 0; h < H; ++h) {
                double const x = pp[rr][h] * shrink;
                pp[rr][h] = (double) (T) (x > 0. ? x : 0.);
              }
            }
          } else {
#pragma unroll
            for(int rr = 0; rr < 4; ++rr) {
#pragma unroll
              for(int h = 0; h < H; ++h) {
                double const x = pp[rr][h];
                pp[rr][h] = (double) (T) (x > thr ? x - thr : (x < -thr ? x + thr : 0.));
              }
            }
          }
#pragma unroll
          for(int rr = 0; rr < 4; ++rr) {
#pragma unroll
            for(int h = 0; h < H; ++h) {
              uint32_t const c = (uint32_t) lane + 32u * h;
              if((uint32_t) rr >= nr || c >= R) { continue; }
              size_t const b = (size_t) (i0 + rr) * R + c;
              double const au = pa[rr][h];
              double const p = pp[rr][h];
              double const d = (double) (T) (ld[rr][h] + (p - au));
              P[b] = (T) p;
              D[b] = (T) d;
              double const pd = p - au, dd = p - lp[rr][h];
              dn = fma(d, d, dn); pn = fma(p, p, pn); pr = fma(pd, pd, pr); dr = fma(dd, dd, dr);
            }
          }
        }
        dn = warp_sum(dn); pn = warp_sum(pn); pr = warp_sum(pr); dr = warp_sum(dr);
        __syncwarp();
        if(pr <= a.inner_tol * pn && dr <= a.inner_tol * dn) { ++it; break; }
      }
      if(lane == 0) { atomicAdd(a.red + RD_CHUNK + mq, (double) it * (double) (c1 - c0)); }
    }
  }

  __device__ void admm_chunked(int mq, double const * Ginv, double const * hb, double rho)
  {
    if(a.R <= 32) { admm_chunked_h<1>(mq, Ginv, hb, rho); }
    else { admm_chunked_h<2>(mq, Ginv, hb, rho); }
  }

  /* ---- column simplex (splatt_colsimp_prox, simplex.cc:113-150, with the
   * vector projection of simplex.cc:28-58), a prox that is not
   * row-separable: every column c of the pre-prox primal P (all rows; the
   * first half stored P = aux - D) becomes max(P - theta_c, 0), theta_c the
   * value at which the column's parts above it sum to 1.  theta_c by
   * Michelot's iteration: round 0 sums and counts every entry, round r the
   * entries above theta_{r-1} = (sum_{r-1} - 1) / count_{r-1}; the rounds
   * stop when a count repeats (the set above theta no longer shrinks) --
   * the support the reference's descending sort and pivot search find, so
   * the same theta up to the order of its sum.  Each round is one grid
   * reduction into a ring of four accumulators (64 sums, 64 counts).  Round
   * r clears round r+1's slot, which is round r-3's: its last readers were
   * round r-2 (theta) and the stop test after round r-2 (counts), both
   * before the barrier that ended round r-1.  A slower block may still run
   * the stop test after round r-1 (reading rounds r-1 and r-2) while round
   * r starts, so a ring of three would clear a slot still being read.
   * Round 0's slot is cleared by the ADMM first half that precedes it. ---- */
  __device__ double * simp_acc(int r) const
  {
    return a.red + RD_SIMP + (r % SB_SIMP_RING) * 128;
  }

  /* theta of round r's accumulator (column c) */
  __device__ double simp_theta(int r, uint32_t c) const
  {
    double const * acc = simp_acc(r);
    return (ldcg(acc + c) - 1.) / ldcg(acc + 64 + c);
  }

  /* round r over this block's rows; r = 0 also clears the ADMM norms of
   * counter k (for colsimp_apply) */
  __device__ void colsimp_round(int mq, int r, int k)
  {
    int const m = a.ns[mq];
    uint32_t const R = a.R;
    if(vb == 0) {
      double * nx = simp_acc(r + 1);
      for(uint32_t e = threadIdx.x; e < 128; e += blockDim.x) { nx[e] = 0.; }
      if(r == 0 && threadIdx.x < 4) { nrm_acc(k)[threadIdx.x] = 0.; }
    }
    double * th = sm + sm_small(R) + 300;
    for(uint32_t c = threadIdx.x; c < R; c += blockDim.x) {
      th[c] = r == 0 ? -INFINITY : simp_theta(r - 1, c);
    }
    __syncthreads();
    uint32_t r0, r1;
    row_range(a.rows[m], vb, nvb, r0, r1);
    int const lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t const c0 = (uint32_t) lane, c1 = c0 + 32;
    double const t0 = c0 < R ? th[c0] : 0., t1 = c1 < R ? th[c1] : 0.;
    double s0 = 0., s1 = 0., n0 = 0., n1 = 0.;
    T const * __restrict__ P = A(m);
    for(uint32_t i = r0 + w; i < r1; i += nw) {
      if(c0 < R) {
        double const x = (double) P[(size_t) i * R + c0];
        if(x > t0) { s0 += x; n0 += 1.; }
      }
      if(c1 < R) {
        double const x = (double) P[(size_t) i * R + c1];
        if(x > t1) { s1 += x; n1 += 1.; }
      }
    }
    block_cols_add(sm + sm_small(R), R, c0, s0, s1, c0 < R, c1 < R, simp_acc(r));
    block_cols_add(sm + sm_small(R), R, c0, n0, n1, c0 < R, c1 < R, simp_acc(r) + 64);
  }

  /* after round r (r >= 1): has every column's set stopped shrinking? */
  __device__ bool colsimp_done(int r) const
  {
    __shared__ int s_same;
    if(threadIdx.x == 0) { s_same = 1; }
    __syncthreads();
    double const * now = simp_acc(r) + 64, * before = simp_acc(r - 1) + 64;
    for(uint32_t c = threadIdx.x; c < a.R; c += blockDim.x) {
      if(ldcg(now + c) < ldcg(before + c)) { s_same = 0; }   /* still shrinking */
    }
    __syncthreads();
    return s_same != 0;
  }

  /* the second half with the column simplex: P = max(P - theta_c, 0) with
   * round r's theta, D += P - aux, and the iteration's four norms into
   * nrm_acc(k) (admm.c:286-301) */
  __device__ void colsimp_apply(int mq, int k, int r)
  {
    int const m = a.ns[mq];
    uint32_t const R = a.R;
    double * th = sm + sm_small(R) + 300;
    for(uint32_t c = threadIdx.x; c < R; c += blockDim.x) { th[c] = simp_theta(r, c); }
    __syncthreads();
    uint32_t r0, r1;
    row_range(a.rows[m], vb, nvb, r0, r1);
    int const lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    T * __restrict__ P = A(m);
    T * __restrict__ D = Dm(m);
    T const * __restrict__ AU = AUX();
    T const * __restrict__ IN = INIT();
    double dn = 0., pn = 0., pr = 0., dr = 0.;
    for(uint32_t i = r0 + w; i < r1; i += nw) {
      for(uint32_t c = (uint32_t) lane; c < R; c += 32) {
        size_t const b = (size_t) i * R + c;
        double const x = (double) P[b] - th[c];
        double const p = (double) (T) (x > 0. ? x : 0.);
        double const au = (double) AU[b];
        double const d = (double) (T) ((double) D[b] + p - au);
        double const pd = p - au, dd = p - (double) IN[b];
        P[b] = (T) p;
        D[b] = (T) d;
        dn = fma(d, d, dn); pn = fma(p, p, pn); pr = fma(pd, pd, pr); dr = fma(dd, dd, dr);
      }
    }
    dn = warp_sum(dn); pn = warp_sum(pn); pr = warp_sum(pr); dr = warp_sum(dr);
    double * part = sm + sm_small(R) + 372;              /* 4 x warps (<= 32) */
    if(lane == 0) { part[4 * w] = dn; part[4 * w + 1] = pn; part[4 * w + 2] = pr; part[4 * w + 3] = dr; }
    __syncthreads();
    if(threadIdx.x < 4) {
      double acc = 0.;
      for(int ww = 0; ww < nw; ++ww) { acc += part[4 * ww + threadIdx.x]; }
      atomicAdd(nrm_acc(k) + threadIdx.x, acc);
    }
    __syncthreads();
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

  /* The same test (fused path) with the next step's column norms cn(k+1)
   * fetched in the same round trip into the shared slots admm_step reads:
   * one L2 latency and one block barrier per iteration instead of two. */
  __device__ bool admm_converged_stage(int k)
  {
    uint32_t const R = a.R;
    double * cn = sm + sm_small(R) + 128;
    double * nr = sm + sm_small(R) + 264;
    uint32_t const t = threadIdx.x;
    if(t < R) { cn[t] = sqrt(ldcg(cn_acc(k + 1) + t)); }
    else if(t < R + 4) { nr[t - R] = ldcg(nrm_acc(k) + (t - R)); }
    __syncthreads();
    return (nr[2] <= a.inner_tol * nr[1]) && (nr[3] <= a.inner_tol * nr[0]);
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
  size_t a = (size_t) sm_xs(R) + (size_t) (ST_THREADS_MAX / 32) * 4 * SB_XS_STRIDE;
  size_t b = (size_t) 64 * R;
  return (a > b ? a : b) * sizeof(double);
}

/* ---- PLAIN executor: one phase per launch ---- */
template <typename T>
__global__ void __launch_bounds__(ST_THREADS_FUSED, 1)
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
  case PH_GRAM: p.gram(mq, false); break;
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
  case PH_ADMM_CHUNKED:
    p.mode_setup(mq, Ginv, hb);
    p.admm_chunked(mq, Ginv, hb, sm[sm_small(R) + 500]);
    break;
  case PH_MODE_FINISH: p.mode_finish(mq, flag, extra); break;
  case PH_EPILOGUE: p.epilogue(flag); break;
  case PH_COLSIMP_ROUND: p.colsimp_round(mq, flag, k); break;
  case PH_COLSIMP_APPLY: p.colsimp_apply(mq, k, flag); break;
  default: break;
  }
}

/* ---- FUSED executor: one slice of one stream on a group of `nvb` blocks
 * (the whole grid for a single stream, a slice of it in a batch); phases are
 * separated by the stream's own bounded group barrier ---- */
template <typename T, bool NN = true>
__device__ void run_slice(StreamArgs const & a, unsigned vb, unsigned nvb, double * sm)
{
  Ph<T, NN> p{a, vb, nvb, sm};
  uint32_t const R = a.R;
  double * Ginv = sm + R * R;
  double * hb = sm + 2 * R * R;
#define SB_BAR() do { if(!grid_barrier(a.bar, a.status, nvb)) { return; } } while(0)

  p.clear_accumulators();
  SB_BAR();
  /* prologue (grow_mats): Grams of the grown factors, then on the first
   * slice the column normalisation (after the Gram, as the reference does) */
  for(int q = 0; q < a.nns; ++q) { p.gram(q, true); }
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
  int chunk_prev[8] = {0, 0, 0, 0, 0, 0, 0, 0};
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
      if(NN && a.prox[a.ns[q]] == SB_PROX_COLSIMP) {
        /* single-chunk ADMM with the column simplex: first half, the
         * threshold rounds (a grid barrier each), second half, test */
        p.admm_first(q, true, k, Ginv, hb, rho);
        SB_BAR();
        int it = 0;
        while(true) {
          int r = 0;
          for(; r < SB_SIMP_MAX_ROUNDS; ++r) {
            p.colsimp_round(q, r, k);
            SB_BAR();
            if(r > 0 && p.colsimp_done(r)) { break; }
          }
          if(r == SB_SIMP_MAX_ROUNDS) { r = SB_SIMP_MAX_ROUNDS - 1; }
          p.colsimp_apply(q, k, r);
          SB_BAR();
          bool const conv = p.admm_converged(k);
          ++it;
          k += 1;
          if(conv || it >= a.max_inner) { break; }
          p.admm_first(q, false, k, Ginv, hb, rho);
          SB_BAR();
        }
        inner_total += it;
        if(vb == 0 && threadIdx.x == 0) {
          a.status[4 + q] = it + (outer > 0 ? a.status[4 + q] : 0);
        }
        uint32_t const next_rows = (q + 1 < a.nns) ? a.rows[a.ns[q + 1]] : 0u;
        p.mode_finish(q, outer, next_rows);
        SB_BAR();
        continue;
      }
      if(NN && SB_PROX_CHUNKED(a.prox[a.ns[q]])) {
        /* row-separable prox: warp-local chunks, one barrier */
        p.admm_chunked(q, Ginv, hb, rho);
        SB_BAR();
        int const cum = (int) llrint(ldcg(a.red + RD_CHUNK + q) / (double) a.rows[a.ns[q]]);
        inner_total += cum - chunk_prev[q];
        chunk_prev[q] = cum;
        if(vb == 0 && threadIdx.x == 0) { a.status[4 + q] = cum; }
        uint32_t const next_rows = (q + 1 < a.nns) ? a.rows[a.ns[q + 1]] : 0u;
        p.mode_finish(q, outer, next_rows);
        SB_BAR();
        continue;
      }
      p.admm_first(q, true, k, Ginv, hb, rho);
      SB_BAR();
      /* One grid barrier per ADMM iteration: the second half of iteration
       * k and (speculatively) the first half of k+1 touch only this block's
       * rows; when the test after the barrier says k converged, P is
       * restored from init and the speculative accumulators are skipped. */
      int it = 0;
      bool staged = false;
      while(true) {
        bool const last = (it + 1 >= a.max_inner);
        p.admm_step(q, k, !last, Ginv, rho, staged);
        SB_BAR();
        bool const conv = p.admm_converged_stage(k);
        staged = true;
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

template <typename T, bool NN>
__global__ void __launch_bounds__(ST_THREADS_FUSED, 1)
k_stream_fused(StreamArgs const a)
{
  extern __shared__ double sm[];
  run_slice<T, NN>(a, blockIdx.x, gridDim.x, sm);
}

/* ---- SCHEDULED executor: chains of slices (each stream's slices in order)
 * run on fixed groups of g blocks.  A group claims the chain with the most
 * slices left that no group holds, runs that chain's next slice with the
 * fused update (group barrier), releases it and claims again; a stream's
 * slices therefore run in order, one at a time, and a slow slice holds only
 * its own group while the others keep taking work.  A group that finds no
 * claimable chain exits: every chain that still has slices is held by a
 * group that is running, which takes that chain again (or another) when its
 * slice ends, so the launch finishes every chain and no group ever waits on
 * another group's progress. ---- */
struct SchedView {
  int C, heavy, ngroups, cap;
  int * err;
  int const * base;
  int const * len;
  int * next;
  int * busy;
  int const * prio;
  int * mbox;
  unsigned * gbar;
  int const * gstart;
  StreamArgs const * items;
};

__device__ __forceinline__ SchedView sched_view(int * blk)
{
  SchedView v;
  v.C = ldcg(blk);
  v.heavy = ldcg(blk + 1);
  v.ngroups = ldcg(blk + 2);
  v.cap = ldcg(blk + 3);
  v.err = blk + 4;
  v.base = blk + 8;
  v.len = v.base + v.cap;
  v.next = (int *) v.len + v.cap;
  v.busy = v.next + v.cap;
  v.prio = v.busy + v.cap;
  v.mbox = (int *) v.prio + v.cap;
  v.gbar = (unsigned *) (v.mbox + SB_SCHED_MAXG);
  v.gstart = (int const *) (v.gbar + 2 * SB_SCHED_MAXG);
  v.items = (StreamArgs const *) ((char const *) blk + SB_SCHED_HDR_BYTES(v.cap));
  return v;
}

/* warp 0 of a group's first block: claim a chain; lane 0 gets (item, chain)
 * or item -1 when nothing is claimable.  Heavy groups take the chain with
 * the largest work estimate, light groups the smallest (ties: more slices
 * left, then the lower index).  At most 64 lost races, each of which means
 * another group took work, then the group exits. */
__device__ int sched_claim(SchedView const & v, int & chain, bool heavy)
{
  unsigned const lane = threadIdx.x & 31u;
  for(int attempt = 0; attempt < 64; ++attempt) {
    long long best = -1;
    int best_c = -1;
    for(int c = (int) lane; c < v.C; c += 32) {
      int const rem = ldcg(v.len + c) - *(volatile int *) (v.next + c);
      if(rem <= 0 || *(volatile int *) (v.busy + c) != 0) { continue; }
      long long const pr = (long long) ldcg(v.prio + c);
      /* one key, larger is better: work (or its complement), then slices left */
      long long const key = ((heavy ? pr : (0x7fffffffLL - pr)) << 20) + (long long) rem;
      if(key > best) { best = key; best_c = c; }
    }
    for(int o = 16; o > 0; o >>= 1) {
      long long const k2 = __shfl_xor_sync(0xffffffffu, best, o);
      int const c2 = __shfl_xor_sync(0xffffffffu, best_c, o);
      if(k2 > best || (k2 == best && c2 >= 0 && (best_c < 0 || c2 < best_c))) {
        best = k2;
        best_c = c2;
      }
    }
    if(best_c < 0) { return -1; }
    int item = -1;
    if(lane == 0 && atomicCAS(v.busy + best_c, 0, 1) == 0) {
      __threadfence();
      int const n = *(volatile int *) (v.next + best_c);
      if(n < ldcg(v.len + best_c)) {
        item = ldcg(v.base + best_c) + n;
      } else {
        atomicExch(v.busy + best_c, 0);
      }
    }
    item = __shfl_sync(0xffffffffu, item, 0);
    if(item >= 0) { chain = best_c; return item; }
  }
  return -1;
}

template <typename T>
__global__ void __launch_bounds__(ST_THREADS_SCHED, 1)
k_stream_sched(int * blk)
{
  extern __shared__ double sm[];
  __shared__ StreamArgs s_args;
  __shared__ SchedView s_v;            /* kept in SMEM: no registers held */
  __shared__ int s_item, s_chain;      /* across the slice update */
  __shared__ int s_grp, s_g0, s_gs;
  if(threadIdx.x == 0) {
    s_v = sched_view(blk);
    int lo = 0, hi = s_v.ngroups;      /* gstart[lo] <= blockIdx.x < gstart[hi] */
    while(hi - lo > 1) {
      int const mid = (lo + hi) >> 1;
      if(ldcg(s_v.gstart + mid) <= (int) blockIdx.x) { lo = mid; } else { hi = mid; }
    }
    int const g0 = ldcg(s_v.gstart + lo), g1 = ldcg(s_v.gstart + lo + 1);
    s_grp = ((int) blockIdx.x < g1) ? lo : -1;     /* blocks past the last group */
    s_g0 = g0;
    s_gs = g1 - g0;
  }
  __syncthreads();
  int const grp = s_grp;
  if(grp < 0) { return; }
  unsigned const vb = blockIdx.x - (unsigned) s_g0;
  unsigned const gs = (unsigned) s_gs;
  bool const heavy = s_gs >= s_v.heavy;
  for(;;) {
    if(vb == 0 && threadIdx.x < 32) {
      int chain = -1;
      int const item = sched_claim(s_v, chain, heavy);
      if(threadIdx.x == 0) {
        *(volatile int *) (s_v.mbox + grp) = item;
        s_chain = chain;
      }
    }
    if(!grid_barrier(s_v.gbar + 2 * grp, s_v.err, gs)) { return; }
    if(threadIdx.x == 0) { s_item = *(volatile int *) (s_v.mbox + grp); }
    __syncthreads();
    int const item = s_item;
    if(item < 0) { return; }
    static_assert(sizeof(StreamArgs) % 4 == 0, "StreamArgs copied as words");
    uint32_t const * src = (uint32_t const *) (s_v.items + item);
    uint32_t * dst = (uint32_t *) &s_args;
    for(uint32_t i = threadIdx.x; i < sizeof(StreamArgs) / 4; i += blockDim.x) { dst[i] = ldcg(src + i); }
    __syncthreads();
    if(threadIdx.x == 0) { s_args.bar = s_v.gbar + 2 * grp; }
    __syncthreads();
    run_slice<T>(s_args, vb, gs, sm);
    /* every block of the group is done with the slice (and with the mailbox) */
    if(!grid_barrier(s_v.gbar + 2 * grp, s_v.err, gs)) { return; }
    if(vb == 0 && threadIdx.x == 0) {
      int * nx = s_v.next + s_chain;
      *(volatile int *) nx = *(volatile int *) nx + 1;
      __threadfence();
      atomicExch(s_v.busy + s_chain, 0);
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
int sb_stream_threads(void) { return ST_THREADS_FUSED; }

int sb_stream_blocks(uint32_t R, int vt)
{
  size_t const smem = stream_smem(R);
  int nb = 0, dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  /* both instantiations (with and without the non-negative prox) must fit */
  int nb2 = 0;
  if(vt == SB_F64) {
    cudaFuncSetAttribute(k_stream_fused<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_stream_fused<double, false>, ST_THREADS_FUSED, smem);
    cudaFuncSetAttribute(k_stream_fused<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb2, k_stream_fused<double, true>, ST_THREADS_FUSED, smem);
  } else {
    cudaFuncSetAttribute(k_stream_fused<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_stream_fused<float, false>, ST_THREADS_FUSED, smem);
    cudaFuncSetAttribute(k_stream_fused<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb2, k_stream_fused<float, true>, ST_THREADS_FUSED, smem);
  }
  if(nb2 < nb) { nb = nb2; }
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
    k_stream_phase<double><<<nblocks, ST_THREADS_FUSED, smem, stream()>>>(*a, phase, mq, flag, extra, k);
  } else {
    cudaFuncSetAttribute(k_stream_phase<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    k_stream_phase<float><<<nblocks, ST_THREADS_FUSED, smem, stream()>>>(*a, phase, mq, flag, extra, k);
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
  cfg.blockDim = dim3(ST_THREADS_FUSED);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream();
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  bool nn = false;
  for(int q = 0; q < a->nns; ++q) { nn = nn || a->prox[a->ns[q]] != SB_PROX_MAXCOLNORM; }
  if(vt == SB_F64) {
    void (* const k)(StreamArgs) = nn ? k_stream_fused<double, true> : k_stream_fused<double, false>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    SB_TRY(cudaLaunchKernelEx(&cfg, k, *a));
  } else {
    void (* const k)(StreamArgs) = nn ? k_stream_fused<float, true> : k_stream_fused<float, false>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    SB_TRY(cudaLaunchKernelEx(&cfg, k, *a));
  }
  return SB_OK;
}

int sb_stream_sched(int * dblock, int vt, int nblocks, uint32_t Rmax)
{
  size_t const smem = stream_smem(Rmax);
  cudaLaunchConfig_t cfg;
  memset(&cfg, 0, sizeof(cfg));
  cfg.gridDim = dim3((unsigned) nblocks);
  cfg.blockDim = dim3(ST_THREADS_SCHED);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream();
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if(vt == SB_F64) {
    cudaFuncSetAttribute(k_stream_sched<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    SB_TRY(cudaLaunchKernelEx(&cfg, k_stream_sched<double>, dblock));
  } else {
    cudaFuncSetAttribute(k_stream_sched<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    SB_TRY(cudaLaunchKernelEx(&cfg, k_stream_sched<float>, dblock));
  }
  return SB_OK;
}

int sb_graph_capture_sched(void ** graph_exec, void * dst, void const * src_pinned, size_t bytes,
    int vt, int nblocks, uint32_t Rmax)
{
  *graph_exec = nullptr;
  cudaGraph_t g = nullptr;
  cudaStream_t const st = stream();
  SB_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaMemcpyAsync(dst, src_pinned, bytes, cudaMemcpyHostToDevice, st);
  int rc = (e == cudaSuccess) ? sb_stream_sched((int *) dst, vt, nblocks, Rmax) : SB_EDEVICE;
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

int sb_set_wait_deadline_ns(uint64_t ns)
{
  unsigned long long const v = ns ? (unsigned long long) ns : 2000000000ull;
  SB_TRY(cudaMemcpyToSymbolAsync(g_wait_deadline_ns, &v, sizeof(v), 0, cudaMemcpyHostToDevice,
                                 stream()));
  SB_TRY(cudaStreamSynchronize(stream()));
  return SB_OK;
}

} /* extern "C" */
