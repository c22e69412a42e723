/*
 * splatt_oracle.h -- CPU restatement of the SPLATT hot path (TEST
 * INFRASTRUCTURE ONLY).
 *
 * This is the oracle the parity tests check the CUDA path against.  Only the
 * test suite, the smoke check and the bench's CPU-baseline leg load it; the
 * product library never links or calls it.  Each routine cites the reference
 * function whose algorithm it restates (paths relative to the SPLATT source
 * tree).  Types: uint64 indices, double values (the reference's default build).
 *
 * Parity of this restatement is pinned against the compiled reference
 * (oracle/_ref, built by oracle/Makefile) by tests/test_oracle_pins.py and by
 * the committed fixtures under tests/golden/.
 */
#ifndef SPLATT_ORACLE_H
#define SPLATT_ORACLE_H
#include <stdint.h>

#define ORC_MAX_NMODES 8

typedef struct {
  uint64_t nmodes, nnz;
  uint64_t dims[ORC_MAX_NMODES];
  uint64_t dim_perm[ORC_MAX_NMODES];
  uint64_t nfibs[ORC_MAX_NMODES];
  uint64_t * fptr[ORC_MAX_NMODES];   /* levels 0..nmodes-2, nfibs[l]+1 each */
  uint64_t * fids[ORC_MAX_NMODES];   /* levels 0..nmodes-1; fids[0] kept */
  double * vals;
} orc_csf;

/* CSF allocation scheme codes follow splatt_csf_type: 0=ONE, 1=TWO, 2=ALL */
void * orc_csf_alloc(uint64_t nmodes, uint64_t nnz, uint64_t const * dims,
    uint64_t * const * inds, double const * vals, int alloc_type);
uint64_t orc_csf_count(void * h);
orc_csf const * orc_csf_get(void * h, uint64_t t);
int orc_csf_info(void * h, uint64_t t, uint64_t * nfibs, uint64_t * dim_perm);
void orc_csf_level(void * h, uint64_t t, uint64_t level, uint64_t * fptr,
    uint64_t * fids);
void orc_csf_vals(void * h, uint64_t t, double * vals);
void orc_csf_free(void * h);

/* dense tiling (SPLATT_DENSETILE): nthreads index ranges on each of the
 * bottom `tilelevel` levels; tile `tile` of tree `t` */
void * orc_csf_alloc_tiled(uint64_t nmodes, uint64_t nnz, uint64_t const * dims,
    uint64_t * const * inds, double const * vals, int alloc_type,
    uint64_t nthreads, uint64_t tilelevel);
uint64_t orc_tcsf_count(void * h);
uint64_t orc_tcsf_ntiles(void * h, uint64_t t);
void orc_tcsf_info(void * h, uint64_t t, uint64_t tile, uint64_t * nfibs,
    uint64_t * dim_perm);
void orc_tcsf_level(void * h, uint64_t t, uint64_t tile, uint64_t level,
    uint64_t * fptr, uint64_t * fids);
void orc_tcsf_vals(void * h, uint64_t t, uint64_t tile, double * vals);
void orc_tcsf_free(void * h);

void orc_mttkrp(void * h, uint64_t mode, uint64_t ncols, double ** mats,
    double * out);
void orc_mttkrp_coo(uint64_t nmodes, uint64_t nnz, uint64_t const * dims,
    uint64_t * const * inds, double const * vals, uint64_t mode,
    uint64_t ncols, double ** mats, double * out);

double orc_cpd(uint64_t nmodes, uint64_t nnz, uint64_t const * dims,
    uint64_t * const * inds, double const * vals, uint64_t rank,
    uint64_t niters, double tol, int seed, double ** factors, double * lambda,
    double * fit, double * fit_per_iter);

uint64_t orc_stream(uint64_t nmodes, uint64_t nnz, uint64_t const * dims,
    uint64_t * const * inds, double const * vals, uint64_t stream_mode,
    uint64_t rank, double forget, double reg, uint64_t max_its, int seed,
    uint64_t max_slices, double * time_out, double ** factors,
    uint64_t * out_rows, uint64_t * outer_its, double * local_errsq, int prox,
    double prox_mult);

/* the streaming parser's preparation (ParserSimple.cc:13-79): the nonzeros
 * ordered by (stream_mode, the following modes cyclically), every other
 * mode relabelled by first appearance; out arrays hold nnz entries each */
void orc_stream_prepare(uint64_t nmodes, uint64_t nnz, uint64_t const * dims,
    uint64_t * const * inds, double const * vals, uint64_t stream_mode,
    uint64_t * const * out_inds, double * out_vals);

/* one application of an ADMM constraint's proximal operator to the I x R
 * row-major block P: 0 max-column-norm, 1 non-negative max-column-norm,
 * 2 lasso, 3 row simplex, 4 NTF-L1, 5 NTF-Frobenius, 6 column simplex,
 * 7 non-negativity (lambda: the multiplier of 2, 4 and 5) */
void orc_prox(int kind, double * P, uint64_t I, uint64_t R, double lambda, double rho);

/* windowed error^2 of the last k of `nslices` streamed slices against the
 * stream's time rows and current factors (the streaming driver's report) */
double orc_stream_window_errsq(uint64_t nmodes, uint64_t nnz, uint64_t const * dims,
    uint64_t * const * inds, double const * vals, uint64_t stream_mode, uint64_t rank,
    uint64_t nslices, double const * time_rows, double * const * factors,
    uint64_t const * rows, uint64_t k);

#endif
