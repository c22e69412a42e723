/*
 * k_dense.cu -- dense kernels of the CPD step, all FP64 arithmetic.
 *
 * Replaces src/matrix.c: mat_aTa (171-205, dsyrk), mat_form_gram (311-345)
 * with splatt_frob_gram (src/cpd/constraints/frob.c:25-37) / mat_trace +
 * mat_add_diag (154-168, 348-358), mat_cholesky + mat_solve_cholesky
 * (104-151, dpotrf/dpotrs, written here from the textbook algorithm),
 * p_mat_2norm (37-96) and the inner product of cpd_innerprod
 * (src/cpd/cpd.c:490-531).
 *
 * Gram layout follows the reference: R x R row-major, upper triangle valid
 * (the same storage as LAPACK's column-major lower triangle).  The Cholesky
 * factor is returned in that layout too: Lt[i*R + j] = L[j][i] for j >= i.
 * Reductions are two-phase (per-block partials, then one ordered pass), so
 * results are deterministic run to run.
 */
#include "common.cuh"

namespace sb {

constexpr int GRAM_ROWS = 64;     /* rows staged in shared memory per step */

/* partial[b][R*R] = sum over the block's rows of a_i a_i^T (upper part) */
template <typename T>
__global__ void __launch_bounds__(256)
k_gram_partial(T const * __restrict__ A, uint64_t I, uint32_t R, uint32_t ld,
    double * __restrict__ part)
{
  extern __shared__ double sh[];          /* GRAM_ROWS x R */
  uint32_t const npairs = R * (R + 1) / 2;
  /* each thread owns up to 16 (i, j) pairs, strided by blockDim */
  double acc[16];
  uint32_t pi[16], pj[16];
  int np = 0;
  for(uint32_t p = threadIdx.x; p < npairs && np < 16; p += blockDim.x, ++np) {
    /* unrank p -> (i, j), j >= i, row-major over the upper triangle */
    uint32_t i = 0, rem = p;
    while(rem >= R - i) { rem -= R - i; ++i; }
    pi[np] = i;
    pj[np] = i + rem;
    acc[np] = 0.;
  }
  for(uint64_t r0 = (uint64_t) blockIdx.x * GRAM_ROWS; r0 < I;
      r0 += (uint64_t) gridDim.x * GRAM_ROWS) {
    uint32_t const nr = (uint32_t) umin64(GRAM_ROWS, I - r0);
    __syncthreads();
    for(uint32_t e = threadIdx.x; e < nr * R; e += blockDim.x) {
      uint32_t const rr = e / R, cc = e % R;
      sh[rr * R + cc] = (double) A[(r0 + rr) * ld + cc];
    }
    __syncthreads();
    for(int q = 0; q < np; ++q) {
      double s = acc[q];
      uint32_t const i = pi[q], j = pj[q];
      for(uint32_t rr = 0; rr < nr; ++rr) { s = fma(sh[rr * R + i], sh[rr * R + j], s); }
      acc[q] = s;
    }
  }
  double * P = part + (size_t) blockIdx.x * R * R;
  for(int q = 0; q < np; ++q) { P[pi[q] * R + pj[q]] = acc[q]; }
}

__global__ void k_gram_reduce(double const * __restrict__ part, uint32_t nb, uint32_t R,
    double * __restrict__ G)
{
  uint32_t const e = blockIdx.x * blockDim.x + threadIdx.x;
  if(e >= R * R) { return; }
  uint32_t const i = e / R, j = e % R;
  if(j < i) { return; }
  double s = 0.;
  for(uint32_t b = 0; b < nb; ++b) { s += part[(size_t) b * R * R + e]; }
  G[e] = s;
}

/* the Gram pointers, passed by value (no device table to allocate and copy) */
struct GramPtrs { double const * p[SB_MAX_NMODES]; };

/* One CTA: G = Hadamard_{m != skip} grams[m] (upper), diag += add
 * (+ trace/R when add_rho), then in-place Cholesky.  Output Lt (upper). */
__global__ void k_form_gram_chol(GramPtrs const grams, uint32_t ngrams,
    uint32_t skip, uint32_t R, double diag_add, int add_rho, double * __restrict__ Lt,
    double * __restrict__ rho_out, int * __restrict__ status)
{
  extern __shared__ double S[];           /* full symmetric R x R */
  __shared__ double s_rho;
  for(uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) {
    uint32_t i = e / R, j = e % R;
    uint32_t const a = i < j ? i : j, b = i < j ? j : i;   /* upper index */
    double g = 1.;
    for(uint32_t m = 0; m < ngrams; ++m) {
      if(m != skip) { g *= grams.p[m][a * R + b]; }
    }
    S[e] = g;
  }
  __syncthreads();
  if(threadIdx.x == 0) {
    double rho = 0.;
    if(add_rho) {
      for(uint32_t i = 0; i < R; ++i) { rho += S[i * R + i]; }
      rho /= (double) R;
    }
    s_rho = rho;
    if(rho_out) { *rho_out = rho; }
  }
  __syncthreads();
  for(uint32_t i = threadIdx.x; i < R; i += blockDim.x) { S[i * R + i] += diag_add + s_rho; }
  __syncthreads();
  /* right-looking Cholesky on the lower triangle of S, two block barriers
   * per step: every thread takes the pivot, the column below it is scaled
   * (one division per row); then warps take the rows and lanes the columns
   * of the trailing update */
  __shared__ int s_bad;
  if(threadIdx.x == 0) { s_bad = 0; }
  __syncthreads();
  uint32_t const lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for(uint32_t k = 0; k < R; ++k) {
    double const d = S[k * R + k];
    double const piv = sqrt(d > 0. ? d : 1.);
    for(uint32_t i = k + 1 + threadIdx.x; i < R; i += blockDim.x) { S[i * R + k] /= piv; }
    __syncthreads();
    if(threadIdx.x == 0) {
      if(!(d > 0.) && s_bad == 0) { s_bad = (int) k + 1; }
      S[k * R + k] = piv;
    }
    for(uint32_t i = k + 1 + w; i < R; i += nw) {
      double const li = S[i * R + k];
      for(uint32_t j = k + 1 + lane; j <= i; j += 32) { S[i * R + j] -= li * S[j * R + k]; }
    }
    __syncthreads();
  }
  for(uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) {
    uint32_t const i = e / R, j = e % R;
    Lt[e] = (j >= i) ? S[j * R + i] : 0.;
  }
  if(threadIdx.x == 0 && status) { *status = s_bad; }
}

/* Warp per row: y = L^{-1} b, x = L^{-T} y.  Lane r%32 holds element r in
 * slot r/32 (KR slots).  L (upper-stored Lt) staged in shared memory. */
template <typename T, int KR>
__global__ void __launch_bounds__(256)
k_chol_solve(double const * __restrict__ Lt, uint32_t R, T * __restrict__ B,
    uint64_t I, uint32_t ld)
{
  extern __shared__ double L[];
  for(uint32_t e = threadIdx.x; e < R * R; e += blockDim.x) { L[e] = Lt[e]; }
  __syncthreads();
  int const lane = threadIdx.x & 31;
  uint64_t const warp = ((uint64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint64_t const nwarps = ((uint64_t) gridDim.x * blockDim.x) >> 5;
  for(uint64_t row = warp; row < I; row += nwarps) {
    T * b = B + row * ld;
    double x[KR];
#pragma unroll
    for(int k = 0; k < KR; ++k) {
      uint32_t const r = (uint32_t) (k * 32 + lane);
      x[k] = r < R ? (double) b[r] : 0.;
    }
    /* forward: L y = b ; L[r][i] = Lt[i*R + r] */
    for(uint32_t i = 0; i < R; ++i) {
      int const ks = (int) (i >> 5), ow = (int) (i & 31);
      double yi = 0.;
#pragma unroll
      for(int k = 0; k < KR; ++k) { if(k == ks) { yi = x[k]; } }
      yi = __shfl_sync(0xffffffffu, yi, ow) / L[i * R + i];
#pragma unroll
      for(int k = 0; k < KR; ++k) {
        uint32_t const r = (uint32_t) (k * 32 + lane);
        if(r == i) { x[k] = yi; }
        else if(r > i && r < R) { x[k] = fma(-L[i * R + r], yi, x[k]); }
      }
    }
    /* backward: L^T x = y ; L^T[r][i] = L[i][r] = Lt[r*R + i] */
    for(uint32_t ii = R; ii-- > 0; ) {
      int const ks = (int) (ii >> 5), ow = (int) (ii & 31);
      double xi = 0.;
#pragma unroll
      for(int k = 0; k < KR; ++k) { if(k == ks) { xi = x[k]; } }
      xi = __shfl_sync(0xffffffffu, xi, ow) / L[ii * R + ii];
#pragma unroll
      for(int k = 0; k < KR; ++k) {
        uint32_t const r = (uint32_t) (k * 32 + lane);
        if(r == ii) { x[k] = xi; }
        else if(r < ii) { x[k] = fma(-L[r * R + ii], xi, x[k]); }
      }
    }
#pragma unroll
    for(int k = 0; k < KR; ++k) {
      uint32_t const r = (uint32_t) (k * 32 + lane);
      if(r < R) { b[r] = (T) x[k]; }
    }
  }
}

/* column sums of squares (kind 0) or of A*M products (kind 1), partials */
template <typename T>
__global__ void __launch_bounds__(256)
k_colsum_partial(T const * __restrict__ A, T const * __restrict__ M, uint64_t I,
    uint32_t R, uint32_t ld, double * __restrict__ part)
{
  extern __shared__ double red[];         /* blockDim.x/R groups x R */
  uint32_t const c = threadIdx.x % R;
  uint32_t const rows_per = blockDim.x / R;
  uint32_t const rsub = threadIdx.x / R;
  double s = 0.;
  if(rsub < rows_per) {
    for(uint64_t i = (uint64_t) blockIdx.x * rows_per + rsub; i < I;
        i += (uint64_t) gridDim.x * rows_per) {
      double const a = (double) A[i * ld + c];
      s = fma(a, M ? (double) M[i * ld + c] : a, s);
    }
  }
  red[threadIdx.x] = (rsub < rows_per) ? s : 0.;
  __syncthreads();
  if(threadIdx.x < R) {
    double t = 0.;
    for(uint32_t q = 0; q < rows_per; ++q) { t += red[q * R + threadIdx.x]; }
    part[(size_t) blockIdx.x * R + threadIdx.x] = t;
  }
}

/* lambda[r] = sqrt(sum_b part[b][r])  (mode 0) ; or the weighted inner
 * product sum_r w[r] * sum_b part[b][r] into out[0] (mode 1) */
__global__ void k_colsum_final(double const * __restrict__ part, uint32_t nb, uint32_t R,
    int mode, double const * __restrict__ w, double * __restrict__ out)
{
  __shared__ double sh[1024];
  for(uint32_t r = threadIdx.x; r < R; r += blockDim.x) {
    double t = 0.;
    for(uint32_t b = 0; b < nb; ++b) { t += part[(size_t) b * R + r]; }
    if(mode == 0) { out[r] = sqrt(t); } else { sh[r] = t * (w ? w[r] : 1.); }
  }
  if(mode == 1) {
    __syncthreads();
    if(threadIdx.x == 0) {
      double s = 0.;
      for(uint32_t r = 0; r < R; ++r) { s += sh[r]; }
      out[0] = s;
    }
  }
}

template <typename T>
__global__ void k_divcols(T * __restrict__ A, uint64_t I, uint32_t R, uint32_t ld,
    double const * __restrict__ lambda)
{
  uint64_t const e = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(e >= I * R) { return; }
  uint64_t const i = e / R;
  uint32_t const c = (uint32_t) (e % R);
  A[i * ld + c] = (T) ((double) A[i * ld + c] / lambda[c]);
}

static unsigned colsum_blocks(uint64_t I, uint32_t R)
{
  uint32_t const rows_per = 256 / R;
  uint64_t b = (I + rows_per - 1) / rows_per;
  if(b > 148 * 4) { b = 148 * 4; }
  if(b == 0) { b = 1; }
  return (unsigned) b;
}

template <typename T>
static int colsum(T const * A, T const * M, uint64_t I, uint32_t R, uint32_t ld, int mode,
    double const * w, double * out)
{
  if(R > 256) { return SB_EINPUT; }
  unsigned const nb = colsum_blocks(I, R);
  double * part = nullptr;
  int rc = talloc(&part, (size_t) nb * R);
  if(rc) { return rc; }
  k_colsum_partial<T><<<nb, 256, 256 * sizeof(double), stream()>>>(A, M, I, R, ld, part);
  k_colsum_final<<<1, 256, 0, stream()>>>(part, nb, R, mode, w, out);
  tfree(part);
  SB_CHECK_LAUNCH();
  return SB_OK;
}

} /* namespace sb */

using namespace sb;

extern "C" {

int sb_gram(void const * A, int vt, uint64_t I, uint32_t R, uint32_t ld, double * G,
    int precision)
{
  if(R == 0 || R > 128 || ld < R) { return SB_EINPUT; }
  if(precision == SB_GRAM_TF32X3 && vt == SB_F32 && R <= 64) {
    return sb_gram_tc((float const *) A, I, R, ld, G);
  }
  SB_TRY(cudaMemsetAsync(G, 0, (size_t) R * R * sizeof(double), stream()));
  if(I == 0) { return SB_OK; }
  uint64_t nb64 = (I + GRAM_ROWS - 1) / GRAM_ROWS;
  unsigned const nb = (unsigned) (nb64 < 148 * 2 ? nb64 : 148 * 2);
  if(R * (R + 1) / 2 > 256 * 16) { return SB_EINPUT; }
  double * part = nullptr;
  int rc = talloc(&part, (size_t) nb * R * R);
  if(rc) { return rc; }
  size_t const smem = (size_t) GRAM_ROWS * R * sizeof(double);
  if(vt == SB_F64) {
    if(smem > 48 * 1024) {
      cudaFuncSetAttribute(k_gram_partial<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    }
    k_gram_partial<double><<<nb, 256, smem, stream()>>>((double const *) A, I, R, ld, part);
  } else {
    if(smem > 48 * 1024) {
      cudaFuncSetAttribute(k_gram_partial<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    }
    k_gram_partial<float><<<nb, 256, smem, stream()>>>((float const *) A, I, R, ld, part);
  }
  k_gram_reduce<<<blocks_for((uint64_t) R * R, 256), 256, 0, stream()>>>(part, nb, R, G);
  tfree(part);
  SB_CHECK_LAUNCH();
  return SB_OK;
}

int sb_form_gram_chol(double const * const * grams, uint32_t ngrams, uint32_t skip,
    uint32_t R, double diag_add, int add_rho, double * L, double * rho_out, int * status)
{
  if(R == 0 || R > 128 || ngrams > SB_MAX_NMODES) { return SB_EINPUT; }
  GramPtrs gp;
  for(uint32_t m = 0; m < SB_MAX_NMODES; ++m) { gp.p[m] = m < ngrams ? grams[m] : nullptr; }
  size_t const smem = (size_t) R * R * sizeof(double);
  if(smem > 48 * 1024) {
    cudaFuncSetAttribute(k_form_gram_chol, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
  }
  k_form_gram_chol<<<1, 256, smem, stream()>>>(gp, ngrams, skip, R, diag_add, add_rho, L,
      rho_out, status);
  SB_CHECK_LAUNCH();
  return SB_OK;
}

int sb_chol_solve(double const * L, uint32_t R, void * B, int vt, uint64_t I, uint32_t ld)
{
  if(R == 0 || R > 128 || ld < R) { return SB_EINPUT; }
  if(I == 0) { return SB_OK; }
  size_t const smem = (size_t) R * R * sizeof(double);
  uint64_t const warps = I;
  uint64_t nb64 = (warps * 32 + 255) / 256;
  unsigned const nb = (unsigned) (nb64 < 148 * 8 ? nb64 : 148 * 8);
  int const kr = (int) ((R + 31) / 32);
#define SB_SOLVE(T, K)                                                                   \
  do {                                                                                   \
    if(smem > 48 * 1024) {                                                               \
      cudaFuncSetAttribute(k_chol_solve<T, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem); \
    }                                                                                    \
    k_chol_solve<T, K><<<nb, 256, smem, stream()>>>(L, R, (T *) B, I, ld);              \
  } while(0)
  if(vt == SB_F64) {
    if(kr == 1) { SB_SOLVE(double, 1); } else if(kr == 2) { SB_SOLVE(double, 2); } else { SB_SOLVE(double, 4); }
  } else {
    if(kr == 1) { SB_SOLVE(float, 1); } else if(kr == 2) { SB_SOLVE(float, 2); } else { SB_SOLVE(float, 4); }
  }
#undef SB_SOLVE
  SB_CHECK_LAUNCH();
  return SB_OK;
}

int sb_normalize(void * A, int vt, uint64_t I, uint32_t R, uint32_t ld, double * lambda)
{
  int rc;
  if(vt == SB_F64) {
    rc = colsum<double>((double const *) A, nullptr, I, R, ld, 0, nullptr, lambda);
    if(rc) { return rc; }
    if(I) { k_divcols<double><<<blocks_for(I * R, 256), 256, 0, stream()>>>((double *) A, I, R, ld, lambda); }
  } else {
    rc = colsum<float>((float const *) A, nullptr, I, R, ld, 0, nullptr, lambda);
    if(rc) { return rc; }
    if(I) { k_divcols<float><<<blocks_for(I * R, 256), 256, 0, stream()>>>((float *) A, I, R, ld, lambda); }
  }
  SB_CHECK_LAUNCH();
  return SB_OK;
}

int sb_inner(void const * A, void const * M, int vt, uint64_t I, uint32_t R, uint32_t ld,
    double const * lambda, double * out)
{
  if(vt == SB_F64) {
    return colsum<double>((double const *) A, (double const *) M, I, R, ld, 1, lambda, out);
  }
  return colsum<float>((float const *) A, (float const *) M, I, R, ld, 1, lambda, out);
}

} /* extern "C" */
