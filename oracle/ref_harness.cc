/*
 * ref_harness.cc -- test-infrastructure driver for the compiled reference.
 *
 * Linked into oracle/_ref/libsplatt_ref{64,32}.so together with the
 * reference's own objects.  It exposes plain extern "C" entry points (pointers
 * and sizes only) so the Python tests and the bench's reference arm can call
 * the reference's stock routines on in-memory inputs:
 *
 *   ref_csf_*     splatt_csf_alloc          (src/csf.c:695-739)
 *   ref_mttkrp    splatt_mttkrp             (src/mttkrp.c:1775-1828)
 *   ref_mttkrp_coo mttkrp_stream            (src/mttkrp.c:1699-1769)
 *   ref_cpd       splatt_alloc_cpd + splatt_cpd (src/cpd/cpd.c:42-141)
 *   ref_stream    ParserSimple + StreamCPD::compute
 *                 (src/cpd/stream/ParserSimple.cc:13-79,
 *                  src/cpd/stream/StreamCPD.cc:311-571)
 *
 * Nothing here changes the reference's arithmetic; it only marshals arrays.
 * This file is the checker's plumbing and is never part of the product.
 */
extern "C" {
#include "base.h"
#include "csf.h"
#include "sptensor.h"
#include "mttkrp.h"
#include "matrix.h"
#include "io.h"
#include "util.h"
#include "cpd/cpd.h"
}
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>
#include <fcntl.h>
#include <sys/time.h>

#if SPLATT_VAL_TYPEWIDTH == 64
#include "cpd/stream/ParserSimple.hxx"
#include "cpd/stream/StreamCPD.hxx"

/* the NTF regularizations are defined in the library (nonneg_lasso.c:67,
 * nonneg_frob.c:74) but declared only by the CLI (cmd_cpd_constraint.h:89-90) */
extern "C" splatt_error_type splatt_register_ntf_lasso(splatt_cpd_opts * opts,
    splatt_val_t const multiplier, splatt_idx_t const * const modes_included,
    splatt_idx_t const num_modes);
extern "C" splatt_error_type splatt_register_ntf_frob(splatt_cpd_opts * opts,
    splatt_val_t const multiplier, splatt_idx_t const * const modes_included,
    splatt_idx_t const num_modes);

#endif

/* the constraints' proximal operators (src/cpd/constraints/ *.c, simplex.cc),
 * all with the signature of splatt_cpd_constraint::prox_func */
#define REF_PROX(name) extern "C" void name(val_t * primal, idx_t const nrows, \
    idx_t const ncols, idx_t const offset, void * data, val_t const rho, \
    bool const should_parallelize)
REF_PROX(splatt_maxcolnorm_prox);
REF_PROX(splatt_maxcolnorm_nonneg_prox);
REF_PROX(splatt_lasso_prox);
REF_PROX(splatt_rowsimp_prox);
REF_PROX(ntf_lasso_prox);
REF_PROX(nonneg_frob_prox);
REF_PROX(splatt_colsimp_prox);
REF_PROX(splatt_nonneg_prox);
#undef REF_PROX

static double p_wall(void)
{
  struct timeval tv;
  gettimeofday(&tv, NULL);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

static sptensor_t * p_make_tt(idx_t nmodes, idx_t nnz, idx_t const * dims,
    idx_t * const * inds, val_t const * vals)
{
  sptensor_t * tt = tt_alloc(nnz, nmodes);
  for(idx_t m=0; m < nmodes; ++m) {
    tt->dims[m] = dims[m];
    memcpy(tt->ind[m], inds[m], nnz * sizeof(idx_t));
  }
  memcpy(tt->vals, vals, nnz * sizeof(val_t));
  return tt;
}

typedef struct {
  splatt_csf * csf;
  double * opts;
  idx_t ncsf;
} ref_csf_handle;

extern "C" {

int ref_idx_width(void) { return SPLATT_IDX_TYPEWIDTH; }
int ref_val_width(void) { return SPLATT_VAL_TYPEWIDTH; }

/* Build CSF(s) with csf_alloc under the given allocation scheme (0=ONE,
 * 1=TWO, 2=ALL), untiled.  Inputs are copied first because csf_alloc sorts
 * its argument in place. */
void * ref_csf_alloc(idx_t nmodes, idx_t nnz, idx_t const * dims,
    idx_t * const * inds, val_t const * vals, int alloc_type, int nthreads)
{
  omp_set_num_threads(nthreads);
  sptensor_t * tt = p_make_tt(nmodes, nnz, dims, inds, vals);
  ref_csf_handle * h = (ref_csf_handle *) malloc(sizeof(*h));
  h->opts = splatt_default_opts();
  h->opts[SPLATT_OPTION_CSF_ALLOC] = alloc_type;
  h->opts[SPLATT_OPTION_TILE] = SPLATT_NOTILE;
  h->opts[SPLATT_OPTION_NTHREADS] = nthreads;
  h->opts[SPLATT_OPTION_VERBOSITY] = SPLATT_VERBOSITY_NONE;
  h->csf = csf_alloc(tt, h->opts);
  h->ncsf = alloc_type == 0 ? 1 : (alloc_type == 1 ? 2 : nmodes);
  tt_free(tt);
  return h;
}

/* The reference's own .tns / .bin reader (src/io.c: tt_read, per-mode index
 * base detection at 278-345).  Returns the tensor; sizes through the out
 * arguments. */
void * ref_tt_read(char const * path, idx_t * nmodes, idx_t * nnz, idx_t * dims)
{
  sptensor_t * tt = tt_read((char *) path);
  if(tt == NULL) { return NULL; }
  *nmodes = tt->nmodes;
  *nnz = tt->nnz;
  for(idx_t m=0; m < tt->nmodes; ++m) { dims[m] = tt->dims[m]; }
  return tt;
}

void ref_tt_get(void * h, idx_t m, idx_t * ind, val_t * vals)
{
  sptensor_t const * tt = (sptensor_t const *) h;
  if(ind != NULL) { memcpy(ind, tt->ind[m], tt->nnz * sizeof(idx_t)); }
  if(vals != NULL) { memcpy(vals, tt->vals, tt->nnz * sizeof(val_t)); }
}

void ref_tt_free(void * h) { tt_free((sptensor_t *) h); }

/* the reference's factor fill (fill_rand, src/util.c:16-40) after
 * srand(seed), on the process-wide rand() */
void ref_fill_rand(unsigned seed, val_t * vals, idx_t n)
{
  srand(seed);
  fill_rand(vals, n);
}

/* the reference's empty-slice removal (tt_remove_empty, src/sptensor.c:
 * 190-252) on a tensor from ref_tt_read; returns the slices removed.
 * ref_tt_dims / ref_tt_indmap read its dims and local -> global maps after
 * (ref_tt_indmap returns 0 for a mode it left unmapped). */
idx_t ref_tt_remove_empty(void * h) { return tt_remove_empty((sptensor_t *) h); }

void ref_tt_dims(void * h, idx_t * dims)
{
  sptensor_t const * tt = (sptensor_t const *) h;
  for(idx_t m=0; m < tt->nmodes; ++m) { dims[m] = tt->dims[m]; }
}

int ref_tt_indmap(void * h, idx_t m, idx_t * out)
{
  sptensor_t const * tt = (sptensor_t const *) h;
  if(tt->indmap[m] == NULL) { return 0; }
  memcpy(out, tt->indmap[m], tt->dims[m] * sizeof(idx_t));
  return 1;
}

/* the reference's binary writer (tt_write_binary, src/io.c:388-474) on a
 * tensor from ref_tt_read, at this build's index and value widths */
void ref_tt_write_bin(void * h, char const * path)
{
  tt_write_binary((sptensor_t *) h, (char *) path);
}

idx_t ref_csf_count(void * vh) { return ((ref_csf_handle *) vh)->ncsf; }

/* csf_alloc with SPLATT_OPTION_TILE = SPLATT_DENSETILE: `tile_threads`
 * ranges per tiled mode, the bottom `tilelevel` levels tiled
 * (src/csf.c:427-501). */
void * ref_csf_alloc_tiled(idx_t nmodes, idx_t nnz, idx_t const * dims,
    idx_t * const * inds, val_t const * vals, int alloc_type, int tile_threads,
    int tilelevel)
{
  omp_set_num_threads(1);
  sptensor_t * tt = p_make_tt(nmodes, nnz, dims, inds, vals);
  ref_csf_handle * h = (ref_csf_handle *) malloc(sizeof(*h));
  h->opts = splatt_default_opts();
  h->opts[SPLATT_OPTION_CSF_ALLOC] = alloc_type;
  h->opts[SPLATT_OPTION_TILE] = SPLATT_DENSETILE;
  h->opts[SPLATT_OPTION_TILELEVEL] = tilelevel;
  h->opts[SPLATT_OPTION_NTHREADS] = tile_threads;
  h->opts[SPLATT_OPTION_VERBOSITY] = SPLATT_VERBOSITY_NONE;
  h->csf = csf_alloc(tt, h->opts);
  h->ncsf = alloc_type == 0 ? 1 : (alloc_type == 1 ? 2 : nmodes);
  tt_free(tt);
  return h;
}

idx_t ref_csf_ntiles(void * vh, idx_t t) { return ((ref_csf_handle *) vh)->csf[t].ntiles; }

/* nfibs of tile `tile` of tensor t; returns 1 if its root fids is NULL */
int ref_csf_tile_info(void * vh, idx_t t, idx_t tile, idx_t * nfibs, idx_t * tile_dims)
{
  splatt_csf const * c = ((ref_csf_handle *) vh)->csf + t;
  for(idx_t l=0; l < c->nmodes; ++l) {
    nfibs[l] = c->pt[tile].nfibs[l];
    tile_dims[l] = c->tile_dims[l];
  }
  return c->pt[tile].fids[0] == NULL;
}

void ref_csf_tile_level(void * vh, idx_t t, idx_t tile, idx_t level, idx_t * fptr,
    idx_t * fids)
{
  splatt_csf const * c = ((ref_csf_handle *) vh)->csf + t;
  csf_sparsity const * pt = c->pt + tile;
  idx_t const n = pt->nfibs[level];
  if(fptr != NULL && level < c->nmodes - 1 && pt->fptr[level] != NULL) {
    memcpy(fptr, pt->fptr[level], (n + 1) * sizeof(idx_t));
  }
  if(fids != NULL && pt->fids[level] != NULL) {
    memcpy(fids, pt->fids[level], n * sizeof(idx_t));
  }
}

void ref_csf_tile_vals(void * vh, idx_t t, idx_t tile, val_t * vals)
{
  splatt_csf const * c = ((ref_csf_handle *) vh)->csf + t;
  csf_sparsity const * pt = c->pt + tile;
  if(pt->vals != NULL) {
    memcpy(vals, pt->vals, pt->nfibs[c->nmodes - 1] * sizeof(val_t));
  }
}

/* nfibs[l] and dim_perm[l] for tensor t. Returns 1 if the root fids is NULL. */
int ref_csf_info(void * vh, idx_t t, idx_t * nfibs, idx_t * dim_perm)
{
  splatt_csf const * c = ((ref_csf_handle *) vh)->csf + t;
  for(idx_t l=0; l < c->nmodes; ++l) {
    nfibs[l] = c->pt->nfibs[l];
    dim_perm[l] = c->dim_perm[l];
  }
  return c->pt->fids[0] == NULL;
}

void ref_csf_level(void * vh, idx_t t, idx_t level, idx_t * fptr, idx_t * fids)
{
  splatt_csf const * c = ((ref_csf_handle *) vh)->csf + t;
  idx_t const n = c->pt->nfibs[level];
  if(fptr != NULL && level < c->nmodes - 1) {
    memcpy(fptr, c->pt->fptr[level], (n + 1) * sizeof(idx_t));
  }
  if(fids != NULL && c->pt->fids[level] != NULL) {
    memcpy(fids, c->pt->fids[level], n * sizeof(idx_t));
  }
}

void ref_csf_vals(void * vh, idx_t t, val_t * vals)
{
  splatt_csf const * c = ((ref_csf_handle *) vh)->csf + t;
  memcpy(vals, c->pt->vals, c->nnz * sizeof(val_t));
}

val_t ref_csf_frobsq(void * vh) { return csf_frobsq(((ref_csf_handle *) vh)->csf); }

/* splatt_mttkrp on the handle's CSF set; returns wall seconds of the call. */
double ref_mttkrp(void * vh, idx_t mode, idx_t ncols, val_t ** mats,
    val_t * out, int nthreads)
{
  ref_csf_handle * h = (ref_csf_handle *) vh;
  h->opts[SPLATT_OPTION_NTHREADS] = nthreads;
  omp_set_num_threads(nthreads);
  double const t0 = p_wall();
  splatt_mttkrp(mode, ncols, h->csf, mats, out, h->opts);
  return p_wall() - t0;
}

void ref_csf_free(void * vh)
{
  ref_csf_handle * h = (ref_csf_handle *) vh;
  csf_free(h->csf, h->opts);
  splatt_free_opts(h->opts);
  free(h);
}

/* COO MTTKRP, the reference's streaming kernel and test gold. */
void ref_mttkrp_coo(idx_t nmodes, idx_t nnz, idx_t const * dims,
    idx_t * const * inds, val_t const * vals, idx_t mode, idx_t ncols,
    val_t ** mats, val_t * out, int nthreads)
{
  omp_set_num_threads(nthreads);
  sptensor_t * tt = p_make_tt(nmodes, nnz, dims, inds, vals);
  matrix_t * mptr[MAX_NMODES + 1];
  for(idx_t m=0; m < nmodes; ++m) {
    mptr[m] = mat_mkptr(mats[m], dims[m], ncols, 1);
  }
  mptr[MAX_NMODES] = mat_mkptr(out, dims[mode], ncols, 1);
  mttkrp_stream(tt, mptr, mode);
  for(idx_t m=0; m < nmodes; ++m) { free(mptr[m]); }
  free(mptr[MAX_NMODES]);
  tt_free(tt);
}

/* Plain CPD-ALS exactly as `splatt cpd` runs it: default (TWOMODE, untiled)
 * CSF, srand(seed) then splatt_alloc_cpd (fill_rand), splatt_cpd.
 * factors[m] must hold dims[m]*rank values.  Returns wall seconds of
 * splatt_cpd alone. */
double ref_cpd(idx_t nmodes, idx_t nnz, idx_t const * dims,
    idx_t * const * inds, val_t const * vals, idx_t rank, idx_t niters,
    double tol, int seed, int nthreads, val_t ** factors, val_t * lambda,
    double * fit)
{
  omp_set_num_threads(nthreads);
  sptensor_t * tt = p_make_tt(nmodes, nnz, dims, inds, vals);
  double * opts = splatt_default_opts();
  opts[SPLATT_OPTION_NTHREADS] = nthreads;
  opts[SPLATT_OPTION_VERBOSITY] = SPLATT_VERBOSITY_NONE;
  splatt_csf * csf = csf_alloc(tt, opts);
  tt_free(tt);

  srand(seed);
  splatt_kruskal * k = splatt_alloc_cpd(csf, rank);
  splatt_cpd_opts * copts = splatt_alloc_cpd_opts();
  copts->max_iterations = niters;
  copts->tolerance = tol;
  splatt_global_opts * gopts = splatt_alloc_global_opts();
  gopts->num_threads = nthreads;
  gopts->verbosity = SPLATT_VERBOSITY_NONE;

  double const t0 = p_wall();
  splatt_cpd(csf, rank, copts, gopts, k);
  double const secs = p_wall() - t0;

  for(idx_t m=0; m < nmodes; ++m) {
    memcpy(factors[m], k->factors[m], dims[m] * rank * sizeof(val_t));
  }
  memcpy(lambda, k->lambda, rank * sizeof(val_t));
  *fit = k->fit;

  splatt_free_cpd(k);
  splatt_free_cpd_opts(copts);
  splatt_free_global_opts(gopts);
  csf_free(csf, opts);
  splatt_free_opts(opts);
  return secs;
}

#if SPLATT_VAL_TYPEWIDTH == 64
/*
 * Streaming CPD exactly as `splatt cpd X.bin --stream=M --reg=frob,L,M` runs
 * it (con 1: `--con=nonneg --reg=frob,L,M`; con 2: `--reg=l1,c --reg=frob,L,M`;
 * con 3: `--con=rowsimp --reg=frob,L,M`).  The tensor is written to `binpath` in the reference's .bin format and
 * read back by ParserSimple (which sorts by time and relabels the other modes
 * by first appearance).  The reference prints per-batch lines to stdout; they
 * are captured to `logpath` and parsed for the per-batch seconds.
 *
 * Outputs: time_out (nslices x rank, row t = the time vector of slice t),
 * factors[m] for every non-streamed m (rows in relabeled order, up to
 * dims[m] rows; the number of rows is written to out_rows[m]),
 * batch_secs[t].  Returns the number of slices.
 */
idx_t ref_stream(idx_t nmodes, idx_t nnz, idx_t const * dims,
    idx_t * const * inds, val_t const * vals, idx_t stream_mode, idx_t rank,
    double forget, double reg, idx_t max_its, int seed, int nthreads,
    char const * binpath, char const * logpath, val_t * time_out,
    val_t ** factors, idx_t * out_rows, double * batch_secs,
    double * local_err, int con, double con_mult)
{
  omp_set_num_threads(nthreads);
  sptensor_t * tt = p_make_tt(nmodes, nnz, dims, inds, vals);
  tt_write_binary(tt, binpath);
  tt_free(tt);

  splatt_cpd_opts * copts = splatt_alloc_cpd_opts();
  copts->max_iterations = max_its;
  idx_t sm = stream_mode;
  if(con) {
    /* con 1: `--con=nonneg --reg=frob,L,M`; con 2: `--reg=l1,con_mult
     * --reg=frob,L,M`; con 3 `--con=rowsimp`; con 4 `--reg=ntf-l1,con_mult`;
     * con 5 `--reg=ntf-frob,con_mult`; con 6 `--con=colsimp`.  The first registers on every mode (an
     * empty mode list means all, cmd_cpd.c:46-56), then frob replaces it on
     * M. */
    idx_t all[SPLATT_MAX_NMODES];
    for(idx_t m=0; m < SPLATT_MAX_NMODES; ++m) { all[m] = m; }
    if(con == 1) { splatt_register_nonneg(copts, all, SPLATT_MAX_NMODES); }
    else if(con == 3) { splatt_register_rowsimp(copts, all, SPLATT_MAX_NMODES); }
    else if(con == 4) { splatt_register_ntf_lasso(copts, con_mult, all, SPLATT_MAX_NMODES); }
    else if(con == 5) { splatt_register_ntf_frob(copts, con_mult, all, SPLATT_MAX_NMODES); }
    else if(con == 6) { splatt_register_colsimp(copts, all, SPLATT_MAX_NMODES); }
    else { splatt_register_lasso(copts, con_mult, all, SPLATT_MAX_NMODES); }
  }
  splatt_register_frob(copts, reg, &sm, 1);
  splatt_global_opts * gopts = splatt_alloc_global_opts();
  gopts->num_threads = nthreads;
  gopts->verbosity = SPLATT_VERBOSITY_NONE;
  gopts->random_seed = seed;
  srand(seed);

  fflush(stdout);
  int const saved = dup(1);
  int const fd = open(logpath, O_WRONLY | O_CREAT | O_TRUNC, 0644);
  dup2(fd, 1);
  close(fd);

  splatt_kruskal * k = NULL;
  {
    ParserSimple parser(binpath, stream_mode);
    StreamCPD cpd(&parser);
    k = cpd.compute(rank, forget, copts, gopts);
  }
  fflush(stdout);
  dup2(saved, 1);
  close(saved);

  idx_t const nslices = k->dims[stream_mode];
  memcpy(time_out, k->factors[stream_mode], nslices * rank * sizeof(val_t));
  for(idx_t m=0; m < nmodes; ++m) {
    out_rows[m] = k->dims[m];
    if(m != stream_mode && factors[m] != NULL) {
      memcpy(factors[m], k->factors[m], k->dims[m] * rank * sizeof(val_t));
    }
  }

  /* parse "batch %5lu: %7lu nnz (%0.5fs) ... local-1: %+0.5f" */
  FILE * f = fopen(logpath, "r");
  char line[1024];
  while(f && fgets(line, sizeof(line), f)) {
    unsigned long b, n;
    double s;
    if(sscanf(line, "batch %lu: %lu nnz (%lfs)", &b, &n, &s) == 3 &&
        b >= 1 && b <= nslices) {
      batch_secs[b-1] = s;
      char * p = strstr(line, "local-1:");
      if(p && local_err) {
        local_err[b-1] = atof(p + 8);
      }
    }
  }
  if(f) { fclose(f); }

  splatt_free_cpd(k);
  splatt_free_cpd_opts(copts);
  splatt_free_global_opts(gopts);
  return nslices;
}
#endif

/*
 * One application of a constraint's proximal operator to the nrows x ncols
 * row-major block `primal`, by the reference's own routine, called as a
 * single-chunk ADMM calls it (should_parallelize true, which the
 * max-column-norm proxes assert; each output row or column is computed by
 * one thread, so the result does not depend on the thread count).
 * kind: 0 max-column-norm, 1 non-negative max-column-norm, 2 lasso, 3 row
 * simplex, 4 NTF-L1, 5 NTF-Frobenius, 6 column simplex, 7 non-negativity.
 * `lambda` is the multiplier the registration stores in `data` (2, 4, 5).
 * Returns 0, or -1 for an unknown kind.
 */
int ref_prox(int kind, val_t * primal, idx_t nrows, idx_t ncols, val_t lambda, val_t rho)
{
  void (*f)(val_t *, idx_t const, idx_t const, idx_t const, void *, val_t const,
            bool const) = NULL;
  switch(kind) {
  case 0: f = splatt_maxcolnorm_prox; break;
  case 1: f = splatt_maxcolnorm_nonneg_prox; break;
  case 2: f = splatt_lasso_prox; break;
  case 3: f = splatt_rowsimp_prox; break;
  case 4: f = ntf_lasso_prox; break;
  case 5: f = nonneg_frob_prox; break;
  case 6: f = splatt_colsimp_prox; break;
  case 7: f = splatt_nonneg_prox; break;
  default: return -1;
  }
  val_t mult = lambda;
  f(primal, nrows, ncols, 0, &mult, rho, true);
  return 0;
}

} /* extern "C" */
