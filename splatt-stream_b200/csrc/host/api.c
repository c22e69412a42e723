/*
 * api.c -- options, global options, coordinate tensors, constraints.
 *
 * Follows src/opts.c:10-74 (defaults), src/sptensor.c:351-369 (coords),
 * src/cpd/cpd.c:84-114 (cpd options), src/cpd/constraints/constraints.c
 * (constraint registry), frob.c:61-95 and maxcolnorm.c:72-96.
 */
#include "sb_host.h"
#include <time.h>

static int g_inited = 0;

int sb_ensure_init(void)
{
  if(g_inited) { return SB_OK; }
  int rc = sb_init(-1);
  if(rc == SB_OK) { g_inited = 1; }
  return rc;
}

splatt_error_type splatt_b200_init(int device)
{
  if(g_inited) { return SPLATT_SUCCESS; }
  int rc = sb_init(device);
  if(rc == SB_OK) { g_inited = 1; }
  return sb_err(rc);
}

void * splatt_b200_get_stream(void)
{
  sb_ensure_init();
  return sb_get_stream();
}

void splatt_b200_set_stream(void * s)
{
  sb_ensure_init();
  sb_set_stream(s);
}

char const * splatt_b200_error_string(void) { return sb_error_string(); }

int splatt_version_major(void) { return SPLATT_VER_MAJOR; }
int splatt_version_minor(void) { return SPLATT_VER_MINOR; }
int splatt_version_subminor(void) { return SPLATT_VER_SUBMINOR; }

double * splatt_default_opts(void)
{
  double * o = malloc(SPLATT_OPTION_NOPTIONS * sizeof(double));
  for(int i = 0; i < SPLATT_OPTION_NOPTIONS; ++i) { o[i] = SPLATT_VAL_OFF; }
  o[SPLATT_OPTION_TOLERANCE] = 1e-5;
  o[SPLATT_OPTION_REGULARIZE] = 0.;
  o[SPLATT_OPTION_NITER] = 50;
  o[SPLATT_OPTION_VERBOSITY] = SPLATT_VERBOSITY_LOW;
  o[SPLATT_OPTION_CSF_ALLOC] = SPLATT_CSF_TWOMODE;
  o[SPLATT_OPTION_TILE] = SPLATT_NOTILE;
  o[SPLATT_OPTION_PRIVTHRESH] = 0.02;
  o[SPLATT_OPTION_TILELEVEL] = 1;
  o[SPLATT_OPTION_DECOMP] = 2;   /* SPLATT_DECOMP_MEDIUM */
  o[SPLATT_OPTION_COMM] = 0;     /* SPLATT_COMM_ALL2ALL */
  o[SPLATT_OPTION_RANDSEED] = (double) time(NULL);
  /* one "thread": the device does the parallel work */
  o[SPLATT_OPTION_NTHREADS] = 1;
  return o;
}

void splatt_free_opts(double * opts) { free(opts); }

splatt_global_opts * splatt_alloc_global_opts(void)
{
  splatt_global_opts * g = malloc(sizeof(*g));
  g->num_threads = 1;
  g->random_seed = (int) time(NULL);
  g->verbosity = SPLATT_VERBOSITY_NONE;
  return g;
}

void splatt_free_global_opts(splatt_global_opts * opts) { free(opts); }

/* ---- coordinates --------------------------------------------------------- */
splatt_coord * splatt_alloc_coord(splatt_idx_t const num_modes, splatt_idx_t const nnz)
{
  if(num_modes > SPLATT_MAX_NMODES || nnz > SIZE_MAX / sizeof(idx_t)) { return NULL; }
  splatt_coord * c = calloc(1, sizeof(*c));
  if(!c) { return NULL; }
  c->nmodes = num_modes;
  c->nnz = nnz;
  int ok = 1;
  for(idx_t m = 0; m < num_modes; ++m) {
    c->ind[m] = malloc((nnz ? nnz : 1) * sizeof(idx_t));
    ok = ok && c->ind[m] != NULL;
  }
  c->vals = malloc((nnz ? nnz : 1) * sizeof(val_t));
  if(!ok || !c->vals) { splatt_free_coord(c); return NULL; }
  return c;
}

void splatt_free_coord(splatt_coord * c)
{
  if(!c) { return; }
  for(idx_t m = 0; m < c->nmodes; ++m) { free(c->ind[m]); free(c->indmap[m]); }
  free(c->vals);
  free(c);
}

splatt_error_type splatt_coord_load(char const * const fname, splatt_coord * const coord)
{
  splatt_coord * t = sb_read_tensor(fname);
  if(!t) { return SPLATT_ERROR_BADINPUT; }
  *coord = *t;
  free(t);
  return SPLATT_SUCCESS;
}

splatt_idx_t splatt_coord_get_nnz(splatt_coord const * const c) { return c->nnz; }
splatt_idx_t splatt_coord_get_modes(splatt_coord const * const c) { return c->nmodes; }
splatt_idx_t * splatt_coord_get_inds(splatt_coord const * const c, splatt_idx_t const m)
{
  return m < c->nmodes ? c->ind[m] : NULL;
}
splatt_val_t * splatt_coord_get_vals(splatt_coord const * const c) { return c->vals; }

/* ---- CPD options / constraints ------------------------------------------ */
splatt_cpd_constraint * splatt_alloc_constraint(splatt_con_solve_type const type)
{
  splatt_cpd_constraint * c = calloc(1, sizeof(*c));
  c->solve_type = type;
  c->hints.row_separable = false;
  c->hints.sparsity_inducing = false;
  sprintf(c->description, "UNCONSTRAINED");
  return c;
}

void splatt_free_constraint(splatt_cpd_constraint * con)
{
  if(!con) { return; }
  if(con->free_func) { con->free_func(con->data); }
  free(con);
}

void splatt_register_constraint(splatt_cpd_opts * const opts, splatt_idx_t const mode,
    splatt_cpd_constraint * const con)
{
  if(mode >= SPLATT_MAX_NMODES) { return; }
  splatt_free_constraint(opts->constraints[mode]);
  opts->constraints[mode] = con;
}

splatt_cpd_opts * splatt_alloc_cpd_opts(void)
{
  splatt_cpd_opts * o = malloc(sizeof(*o));
  o->tolerance = 1e-5;
  o->max_iterations = 200;
  o->inner_tolerance = 1e-2;
  o->max_inner_iterations = 50;
  for(idx_t m = 0; m < SPLATT_MAX_NMODES; ++m) {
    o->chunk_sizes[m] = 50;
    o->constraints[m] = splatt_alloc_constraint(SPLATT_CON_CLOSEDFORM);
  }
  return o;
}

void splatt_free_cpd_opts(splatt_cpd_opts * opts)
{
  if(!opts) { return; }
  for(idx_t m = 0; m < SPLATT_MAX_NMODES; ++m) { splatt_free_constraint(opts->constraints[m]); }
  free(opts);
}

/* Tikhonov regularisation: Gram diagonal += multiplier (frob.c:25-37).  The
 * device solver reads the multiplier from `data`; gram_func is kept so host
 * callers inspecting the constraint see SPLATT's structure. */
static void sb_frob_gram(val_t * gram, idx_t const N, void * data)
{
  val_t const mult = *(val_t *) data;
  for(idx_t n = 0; n < N; ++n) { gram[n + n * N] += mult; }
}

splatt_error_type splatt_register_frob(splatt_cpd_opts * opts, splatt_val_t const multiplier,
    splatt_idx_t const * const modes_included, splatt_idx_t const num_modes)
{
  for(idx_t i = 0; i < num_modes; ++i) {
    splatt_cpd_constraint * c = splatt_alloc_constraint(SPLATT_CON_CLOSEDFORM);
    c->gram_func = sb_frob_gram;
    c->free_func = free;
    c->hints.row_separable = true;
    sprintf(c->description, "FROBENIUS-REG (%0.1e)", (double) multiplier);
    val_t * m = malloc(sizeof(*m));
    *m = multiplier;
    c->data = m;
    splatt_register_constraint(opts, modes_included[i], c);
  }
  return SPLATT_SUCCESS;
}

/* max-column-norm: ADMM with column normalisation when norm > 1
 * (maxcolnorm.c:32-96).  The prox runs on the device; the host pointer is a
 * marker only. */
static void sb_maxcolnorm_marker(val_t * p, idx_t const a, idx_t const b, idx_t const c,
    void * d, val_t const rho, bool const par)
{
  (void) p; (void) a; (void) b; (void) c; (void) d; (void) rho; (void) par;
}

splatt_error_type splatt_register_maxcolnorm(splatt_cpd_opts * opts,
    splatt_idx_t const * const modes_included, splatt_idx_t const num_modes)
{
  for(idx_t i = 0; i < num_modes; ++i) {
    splatt_cpd_constraint * c = splatt_alloc_constraint(SPLATT_CON_ADMM);
    c->prox_func = sb_maxcolnorm_marker;
    c->hints.row_separable = false;
    c->hints.sparsity_inducing = false;
    sprintf(c->description, "MAX-COL-NORM");
    splatt_register_constraint(opts, modes_included[i], c);
  }
  return SPLATT_SUCCESS;
}

/* non-negativity (nonneg.c:20-85): negatives zeroed.  The streaming driver
 * turns it into the non-negative max-column-norm on its non-streamed modes,
 * as StreamCPD::compute does (src/cpd/stream/StreamCPD.cc:325-337). */
splatt_error_type splatt_register_nonneg(splatt_cpd_opts * opts,
    splatt_idx_t const * const modes_included, splatt_idx_t const num_modes)
{
  for(idx_t i = 0; i < num_modes; ++i) {
    splatt_cpd_constraint * c = splatt_alloc_constraint(SPLATT_CON_ADMM);
    c->prox_func = sb_maxcolnorm_marker;
    c->hints.row_separable = true;
    c->hints.sparsity_inducing = true;
    sprintf(c->description, "NON-NEGATIVE");
    splatt_register_constraint(opts, modes_included[i], c);
  }
  return SPLATT_SUCCESS;
}

/* max-column-norm over the non-negative orthant (maxcolnorm-nonneg.c:32-102):
 * negatives zeroed, then columns with norm > 1 scaled to unit norm */
splatt_error_type splatt_register_maxcolnorm_nonneg(splatt_cpd_opts * opts,
    splatt_idx_t const * const modes_included, splatt_idx_t const num_modes)
{
  for(idx_t i = 0; i < num_modes; ++i) {
    splatt_cpd_constraint * c = splatt_alloc_constraint(SPLATT_CON_ADMM);
    c->prox_func = sb_maxcolnorm_marker;
    c->hints.row_separable = false;
    c->hints.sparsity_inducing = true;
    sprintf(c->description, "NONNEG-MAX-COL-NORM");
    splatt_register_constraint(opts, modes_included[i], c);
  }
  return SPLATT_SUCCESS;
}

/* row simplex (simplex.cc:71-186): every row projected onto the probability
 * simplex, row-separable */
splatt_error_type splatt_register_rowsimp(splatt_cpd_opts * opts,
    splatt_idx_t const * const modes_included, splatt_idx_t const num_modes)
{
  for(idx_t i = 0; i < num_modes; ++i) {
    splatt_cpd_constraint * c = splatt_alloc_constraint(SPLATT_CON_ADMM);
    c->prox_func = sb_maxcolnorm_marker;
    c->hints.row_separable = true;
    c->hints.sparsity_inducing = true;
    sprintf(c->description, "ROW-SIMPLEX");
    splatt_register_constraint(opts, modes_included[i], c);
  }
  return SPLATT_SUCCESS;
}

/* L1 regularisation (lasso.c:32-107): soft threshold at multiplier / rho,
 * row-separable (the ADMM runs in independent row chunks) */
splatt_error_type splatt_register_lasso(splatt_cpd_opts * opts, splatt_val_t const multiplier,
    splatt_idx_t const * const modes_included, splatt_idx_t const num_modes)
{
  for(idx_t i = 0; i < num_modes; ++i) {
    splatt_cpd_constraint * c = splatt_alloc_constraint(SPLATT_CON_ADMM);
    c->prox_func = sb_maxcolnorm_marker;
    c->free_func = free;
    c->hints.row_separable = true;
    c->hints.sparsity_inducing = true;
    sprintf(c->description, "L1-REG (%0.1e)", (double) multiplier);
    val_t * m = malloc(sizeof(*m));
    *m = multiplier;
    c->data = m;
    splatt_register_constraint(opts, modes_included[i], c);
  }
  return SPLATT_SUCCESS;
}

/* NTF regularizations (nonneg_lasso.c:30-100, nonneg_frob.c:31-105): the
 * one-sided threshold at multiplier / rho, and the shrink rho / (multiplier +
 * rho) followed by zeroing negatives; both row-separable.  The reference
 * gives both the description "NTF-L1-REG"; the prox marker distinguishes
 * them here. */
static void sb_ntf_frob_marker(val_t * p, idx_t const a, idx_t const b, idx_t const c,
    void * d, val_t const rho, bool const par)
{
  (void) p; (void) a; (void) b; (void) c; (void) d; (void) rho; (void) par;
}

static splatt_error_type sb_register_ntf(splatt_cpd_opts * opts, splatt_val_t const multiplier,
    splatt_idx_t const * const modes_included, splatt_idx_t const num_modes, int frob)
{
  for(idx_t i = 0; i < num_modes; ++i) {
    splatt_cpd_constraint * c = splatt_alloc_constraint(SPLATT_CON_ADMM);
    c->prox_func = frob ? sb_ntf_frob_marker : sb_maxcolnorm_marker;
    c->free_func = free;
    c->hints.row_separable = true;
    c->hints.sparsity_inducing = true;
    sprintf(c->description, "NTF-L1-REG (%0.1e)", (double) multiplier);
    val_t * m = malloc(sizeof(*m));
    *m = multiplier;
    c->data = m;
    splatt_register_constraint(opts, modes_included[i], c);
  }
  return SPLATT_SUCCESS;
}

splatt_error_type splatt_register_ntf_lasso(splatt_cpd_opts * opts,
    splatt_val_t const multiplier, splatt_idx_t const * const modes_included,
    splatt_idx_t const num_modes)
{
  return sb_register_ntf(opts, multiplier, modes_included, num_modes, 0);
}

splatt_error_type splatt_register_ntf_frob(splatt_cpd_opts * opts,
    splatt_val_t const multiplier, splatt_idx_t const * const modes_included,
    splatt_idx_t const num_modes)
{
  return sb_register_ntf(opts, multiplier, modes_included, num_modes, 1);
}

int sb_con_is_ntf_frob(splatt_cpd_constraint const * c)
{
  return c && c->prox_func == sb_ntf_frob_marker;
}

/* column simplex (simplex.cc:194-217) and column smoothness (smooth.c:
 * 220-245): registered with SPLATT's descriptions and hints; no solver here
 * accepts them yet, so they are refused where they would be used */
splatt_error_type splatt_register_colsimp(splatt_cpd_opts * opts,
    splatt_idx_t const * const modes_included, splatt_idx_t const num_modes)
{
  for(idx_t i = 0; i < num_modes; ++i) {
    splatt_cpd_constraint * c = splatt_alloc_constraint(SPLATT_CON_ADMM);
    c->prox_func = sb_maxcolnorm_marker;
    c->hints.sparsity_inducing = true;
    sprintf(c->description, "COL-SIMPLEX");
    splatt_register_constraint(opts, modes_included[i], c);
  }
  return SPLATT_SUCCESS;
}

splatt_error_type splatt_register_smooth(splatt_cpd_opts * opts, splatt_val_t const multiplier,
    splatt_idx_t const * const modes_included, splatt_idx_t const num_modes)
{
  for(idx_t i = 0; i < num_modes; ++i) {
    splatt_cpd_constraint * c = splatt_alloc_constraint(SPLATT_CON_ADMM);
    c->prox_func = sb_maxcolnorm_marker;
    c->free_func = free;
    sprintf(c->description, "SMOOTH-COL (%0.1e)", (double) multiplier);
    val_t * m = malloc(sizeof(*m));
    *m = multiplier;
    c->data = m;
    splatt_register_constraint(opts, modes_included[i], c);
  }
  return SPLATT_SUCCESS;
}

/* ---- helpers ------------------------------------------------------------- */
void sb_fill_rand(val_t * v, idx_t n)
{
  for(idx_t i = 0; i < n; ++i) {
    val_t x = (val_t) (3.0 * ((val_t) rand() / (val_t) RAND_MAX));
    if(rand() % 2 == 0) { x = -x; }
    v[i] = x;
  }
}

void sb_order_small(idx_t const * dims, idx_t nmodes, idx_t * perm)
{
  for(idx_t m = 0; m < nmodes; ++m) { perm[m] = m; }
  for(idx_t i = 1; i < nmodes; ++i) {
    idx_t x = perm[i];
    idx_t j = i;
    while(j > 0 && dims[perm[j-1]] > dims[x]) { perm[j] = perm[j-1]; --j; }
    perm[j] = x;
  }
}

void sb_order_minusone(idx_t const * dims, idx_t nmodes, idx_t special, idx_t * perm)
{
  idx_t tmp[SPLATT_MAX_NMODES];
  sb_order_small(dims, nmodes, tmp);
  perm[0] = special;
  idx_t k = 1;
  for(idx_t m = 0; m < nmodes; ++m) {
    if(tmp[m] != special) { perm[k++] = tmp[m]; }
  }
}
