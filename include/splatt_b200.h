/*
 * splatt_b200.h -- public C ABI of libsplatt_b200.so, a B200 (sm_100a)
 * implementation of SPLATT's CSF MTTKRP, CPD-ALS and streaming CPD.
 *
 * Drop-in boundary: the entry points below carry the names, argument meaning
 * and error codes of SPLATT's public API; each cites the declaration it
 * replaces (paths inside the SPLATT source tree).  Types follow SPLATT's
 * build-time widths: SPLATT_IDX_TYPEWIDTH / SPLATT_VAL_TYPEWIDTH (64 by
 * default; libsplatt_b200_w32.so is the 32/32 build).  Host arrays in,
 * host arrays out; device memory is owned by the returned handles.
 *
 * Extensions (splatt_b200_* names) expose device-resident and streaming
 * entry points with no counterpart in SPLATT; each says so.
 */
#ifndef SPLATT_B200_H
#define SPLATT_B200_H

#include <inttypes.h>
#include <stdbool.h>
#include <stddef.h>
#include <float.h>

/* ---- types (include/splatt/types_config.h:34-87) ------------------------ */
#ifndef SPLATT_IDX_TYPEWIDTH
#define SPLATT_IDX_TYPEWIDTH 64
#endif
#ifndef SPLATT_VAL_TYPEWIDTH
#define SPLATT_VAL_TYPEWIDTH 64
#endif

#if SPLATT_IDX_TYPEWIDTH == 32
typedef uint32_t splatt_idx_t;
#define SPLATT_IDX_MAX UINT32_MAX
#define SPLATT_PF_IDX PRIu32
#else
typedef uint64_t splatt_idx_t;
#define SPLATT_IDX_MAX UINT64_MAX
#define SPLATT_PF_IDX PRIu64
#endif

#if SPLATT_VAL_TYPEWIDTH == 32
typedef float splatt_val_t;
#else
typedef double splatt_val_t;
#endif

#define SPLATT_MAX_NMODES ((splatt_idx_t) 8)
/* include/splatt/constants.h: option value meaning "not set" */
#define SPLATT_VAL_OFF (-DBL_MAX)

/* ---- enums (include/splatt/types_config.h:105-176) ---------------------- */
typedef enum {
  SPLATT_OPTION_NTHREADS,
  SPLATT_OPTION_TOLERANCE,
  SPLATT_OPTION_REGULARIZE,
  SPLATT_OPTION_NITER,
  SPLATT_OPTION_VERBOSITY,
  SPLATT_OPTION_RANDSEED,
  SPLATT_OPTION_CSF_ALLOC,
  SPLATT_OPTION_TILE,
  SPLATT_OPTION_TILELEVEL,
  SPLATT_OPTION_PRIVTHRESH,
  SPLATT_OPTION_DECOMP,
  SPLATT_OPTION_COMM,
  SPLATT_OPTION_NOPTIONS
} splatt_option_type;

typedef enum {
  SPLATT_SUCCESS = 1,
  SPLATT_ERROR_BADINPUT,
  SPLATT_ERROR_NOMEMORY,
  /* extension: a CUDA call failed for a reason other than memory */
  SPLATT_ERROR_DEVICE
} splatt_error_type;

typedef enum {
  SPLATT_VERBOSITY_NONE,
  SPLATT_VERBOSITY_LOW,
  SPLATT_VERBOSITY_HIGH,
  SPLATT_VERBOSITY_MAX
} splatt_verbosity_type;

typedef enum {
  SPLATT_NOTILE,
  SPLATT_DENSETILE,
  SPLATT_SYNCTILE,
  SPLATT_COOPTILE
} splatt_tile_type;

typedef enum {
  SPLATT_CSF_ONEMODE,
  SPLATT_CSF_TWOMODE,
  SPLATT_CSF_ALLMODE
} splatt_csf_type;

/* ---- global options (include/splatt/global_options.h:18-24) ------------- */
typedef struct {
  int num_threads;
  splatt_verbosity_type verbosity;
  int random_seed;
} splatt_global_opts;

/* ---- coordinate tensor (src/sptensor.h:16-64, include/splatt/coord.h) --- */
typedef struct _splatt_coord {
  splatt_idx_t nmodes;
  splatt_idx_t dims[8];
  splatt_idx_t nnz;
  splatt_idx_t * ind[8];
  splatt_val_t * vals;
  int tiled;
  splatt_idx_t * indmap[8];
} splatt_coord;

/* ---- CSF (src/csf.h:28-94) ---------------------------------------------- */
typedef struct {
  splatt_idx_t nfibs[8];
  splatt_idx_t * fptr[8];
  splatt_idx_t * fids[8];
  splatt_val_t * vals;
} csf_sparsity;

typedef struct _splatt_csf {
  splatt_idx_t nnz;
  splatt_idx_t nmodes;
  splatt_idx_t dims[8];
  splatt_idx_t dim_perm[8];
  splatt_idx_t dim_iperm[8];
  splatt_tile_type which_tile;
  splatt_idx_t ntiles;
  splatt_idx_t ntiled_modes;
  splatt_idx_t tile_dims[8];
  csf_sparsity * pt;
  /* B200: the device copy of this tree (fptr/fids as uint32, root ids kept) */
  void * dev;
} splatt_csf;

/* ---- CPD (include/splatt/cpd.h:26-150, src/cpd/cpd.h:37-56) ------------- */
typedef struct {
  bool row_separable;
  bool sparsity_inducing;
} splatt_con_hints;

typedef enum {
  SPLATT_CON_CLOSEDFORM,
  SPLATT_CON_ADMM
} splatt_con_solve_type;

typedef struct {
  splatt_con_solve_type solve_type;
  splatt_con_hints hints;
  void * data;
  char description[256];
  void (* init_func)(splatt_val_t *, splatt_idx_t const, splatt_idx_t const, void *);
  void (* gram_func)(splatt_val_t *, splatt_idx_t const, void *);
  void (* prox_func)(splatt_val_t *, splatt_idx_t const, splatt_idx_t const,
      splatt_idx_t const, void *, splatt_val_t const, bool const);
  void (* clsd_func)(splatt_val_t *, splatt_idx_t const, splatt_idx_t const, void *);
  void (* post_func)(splatt_val_t *, splatt_idx_t const, splatt_idx_t const, void *);
  void (* free_func)(void *);
} splatt_cpd_constraint;

typedef struct {
  splatt_val_t tolerance;
  splatt_idx_t max_iterations;
  splatt_val_t inner_tolerance;
  splatt_idx_t max_inner_iterations;
  splatt_cpd_constraint * constraints[8];
  splatt_idx_t chunk_sizes[8];
} splatt_cpd_opts;

typedef struct _splatt_kruskal {
  splatt_idx_t rank;
  splatt_val_t * factors[8];
  splatt_val_t * lambda;
  splatt_idx_t nmodes;
  splatt_idx_t dims[8];
  double fit;
} splatt_kruskal;

/* ---- MTTKRP workspace (include/splatt/api_kernels.h:22-67) -------------- */
typedef struct {
  splatt_idx_t num_csf;
  splatt_idx_t mode_csf_map[8];
  splatt_idx_t num_threads;
  splatt_idx_t * tile_partition[8];
  splatt_idx_t * tree_partition[8];
  bool is_privatized[8];
  splatt_val_t ** privatize_buffer;
  double reduction_time;
} splatt_mttkrp_ws;

#ifdef __cplusplus
extern "C" {
#endif

/* ===== version (include/splatt/api_version.h:18-63) ====================== */
/* The SPLATT API version this library is a drop-in for. */
#define SPLATT_VER_MAJOR     2
#define SPLATT_VER_MINOR     0
#define SPLATT_VER_SUBMINOR  0
int splatt_version_major(void);
int splatt_version_minor(void);
int splatt_version_subminor(void);

/* ===== options (include/splatt/api_options.h:37,43; global_options.h) ==== */
/* The defaults are SPLATT's (src/opts.c:14-75), except SPLATT_OPTION_NTHREADS
 * and splatt_global_opts::num_threads, which are 1 here (SPLATT: the OpenMP
 * thread count): the device does the parallel work.  The only result that
 * depends on it is the tile count of SPLATT_DENSETILE, so a caller relying on
 * SPLATT's default tiling sets SPLATT_OPTION_NTHREADS itself. */
double * splatt_default_opts(void);                          /* api_options.h:37 */
void splatt_free_opts(double * opts);                        /* api_options.h:43 */
splatt_global_opts * splatt_alloc_global_opts(void);         /* global_options.h:40 */
void splatt_free_global_opts(splatt_global_opts * opts);     /* global_options.h:48 */

/* ===== coordinate tensors (include/splatt/coord.h:53-121) ================= */
splatt_coord * splatt_alloc_coord(splatt_idx_t const num_modes, splatt_idx_t const nnz);
void splatt_free_coord(splatt_coord * coord);
splatt_error_type splatt_coord_load(char const * const fname, splatt_coord * const coord);
splatt_idx_t splatt_coord_get_nnz(splatt_coord const * const coord);
splatt_idx_t splatt_coord_get_modes(splatt_coord const * const coord);
splatt_idx_t * splatt_coord_get_inds(splatt_coord const * const coord, splatt_idx_t const mode);
splatt_val_t * splatt_coord_get_vals(splatt_coord const * const coord);

/* ===== CSF (include/splatt/csf.h:55-102, src/csf.h:108-186) ============== */
/* csf.h:55-59 -- read .tns/.bin, drop empty slices, build CSF(s) on device */
splatt_error_type splatt_csf_load(char const * const fname, splatt_idx_t * nmodes,
    splatt_csf ** tensors, double const * const options);
/* csf.h:83-89 (declared under #if 0 in SPLATT; defined here).  Allocation
 * scheme from options[SPLATT_OPTION_CSF_ALLOC]; options[SPLATT_OPTION_TILE]
 * SPLATT_NOTILE or SPLATT_DENSETILE (src/csf.c:427-501: the bottom
 * SPLATT_OPTION_TILELEVEL levels cut into SPLATT_OPTION_NTHREADS index ranges,
 * one CSF per tile in `pt[0..ntiles)`, root ids kept when ntiles > 1;
 * TWOMODE's second tree untiled).  Other tile schemes: SPLATT_ERROR_BADINPUT. */
splatt_error_type splatt_csf_convert(splatt_idx_t const nmodes, splatt_idx_t const nnz,
    splatt_idx_t ** const inds, splatt_val_t * const vals, splatt_csf ** tensors,
    double const * const options);
/* csf.h:100-102 */
void splatt_free_csf(splatt_csf * tensors, double const * const options);
/* src/csf.h:108-121 (csf_alloc): sorts tt in place, as SPLATT does */
splatt_csf * splatt_csf_alloc(splatt_coord * const tt, double const * const opts);
/* src/csf.h:148-152 (csf_free) */
void splatt_csf_free(splatt_csf * const csf, double const * const opts);
/* src/csf.h:183-186 (csf_frobsq) */
splatt_val_t splatt_csf_frobsq(splatt_csf const * const tensor);

/* ===== MTTKRP (include/splatt/api_kernels.h:98-119) ====================== */
int splatt_mttkrp(splatt_idx_t const mode, splatt_idx_t const ncolumns,
    splatt_csf const * const tensors, splatt_val_t ** matrices,
    splatt_val_t * const matout, double const * const options);
splatt_mttkrp_ws * splatt_mttkrp_alloc_ws(splatt_csf const * const tensors,
    splatt_idx_t const ncolumns, double const * const options);
void splatt_mttkrp_free_ws(splatt_mttkrp_ws * const ws);

/* ===== CPD (include/splatt/cpd.h:173-380) ================================ */
splatt_kruskal * splatt_alloc_cpd(splatt_csf const * const csf, splatt_idx_t rank);
void splatt_free_cpd(splatt_kruskal * factored);
splatt_error_type splatt_cpd(splatt_csf const * const tensor, splatt_idx_t rank,
    splatt_cpd_opts const * const cpd_opts, splatt_global_opts const * const global_opts,
    splatt_kruskal * factored);
splatt_cpd_opts * splatt_alloc_cpd_opts(void);
void splatt_free_cpd_opts(splatt_cpd_opts * opts);
splatt_cpd_constraint * splatt_alloc_constraint(splatt_con_solve_type const type);
void splatt_free_constraint(splatt_cpd_constraint * con);
void splatt_register_constraint(splatt_cpd_opts * const opts, splatt_idx_t const mode,
    splatt_cpd_constraint * const con);
splatt_error_type splatt_register_frob(splatt_cpd_opts * opts, splatt_val_t const multiplier,
    splatt_idx_t const * const modes_included, splatt_idx_t const num_modes);
splatt_error_type splatt_register_maxcolnorm(splatt_cpd_opts * opts,
    splatt_idx_t const * const modes_included, splatt_idx_t const num_modes);
/* include/splatt/cpd.h:245-265.  ADMM constraints run on the streaming
 * path's non-streamed modes (splatt_cpd returns SPLATT_ERROR_BADINPUT for
 * them). */
splatt_error_type splatt_register_maxcolnorm_nonneg(splatt_cpd_opts * opts,
    splatt_idx_t const * const modes_included, splatt_idx_t const num_modes);
splatt_error_type splatt_register_nonneg(splatt_cpd_opts * opts,
    splatt_idx_t const * const modes_included, splatt_idx_t const num_modes);
/* include/splatt/cpd.h:279-282 */
splatt_error_type splatt_register_rowsimp(splatt_cpd_opts * opts,
    splatt_idx_t const * const modes_included, splatt_idx_t const num_modes);
/* include/splatt/cpd.h:332-335 */
splatt_error_type splatt_register_lasso(splatt_cpd_opts * opts, splatt_val_t const multiplier,
    splatt_idx_t const * const modes_included, splatt_idx_t const num_modes);
/* The NTF regularizations of the CLI's `--reg=ntf-l1,L` and
 * `--reg=ntf-frob,L` (src/cmds/cmd_cpd_constraint.h:89-90, 145-146; defined
 * in nonneg_lasso.c:67-100 and nonneg_frob.c:74-105).  Both are described
 * "NTF-L1-REG (L)", as there. */
splatt_error_type splatt_register_ntf_lasso(splatt_cpd_opts * opts,
    splatt_val_t const multiplier, splatt_idx_t const * const modes_included,
    splatt_idx_t const num_modes);
splatt_error_type splatt_register_ntf_frob(splatt_cpd_opts * opts,
    splatt_val_t const multiplier, splatt_idx_t const * const modes_included,
    splatt_idx_t const num_modes);
/* include/splatt/cpd.h:297-300 and 349-353: registered as in SPLATT
 * ("COL-SIMPLEX", "SMOOTH-COL (L)"; simplex.cc:194-217, smooth.c:220-245).
 * splatt_cpd_stream runs the column simplex on a non-streamed mode
 * (`--con=colsimp`); splatt_cpd returns SPLATT_ERROR_BADINPUT for both, and
 * splatt_cpd_stream for smooth. */
splatt_error_type splatt_register_colsimp(splatt_cpd_opts * opts,
    splatt_idx_t const * const modes_included, splatt_idx_t const num_modes);
splatt_error_type splatt_register_smooth(splatt_cpd_opts * opts, splatt_val_t const multiplier,
    splatt_idx_t const * const modes_included, splatt_idx_t const num_modes);

/* ===== streaming CPD (src/cpd/stream.h:24-30) ============================= */
/* Streams `filename` (.tns/.bin) over `stream_mode` exactly like
 * `splatt cpd FILE --stream=MODE+1 --reg=frob,L,MODE+1`; writes mode%d.mat.
 * The streamed mode takes FROBENIUS-REG or nothing; a non-streamed mode
 * takes nothing / MAX-COL-NORM (max-column-norm prox), NON-NEGATIVE /
 * NONNEG-MAX-COL-NORM (the non-negative one, as `--con=nonneg`), L1-REG
 * (`--reg=l1,L`), ROW-SIMPLEX (`--con=rowsimp`), NTF-L1-REG (from
 * splatt_register_ntf_lasso or _ntf_frob, `--reg=ntf-l1,L` / `ntf-frob,L`)
 * or COL-SIMPLEX (`--con=colsimp`); L1, the row simplex and the NTF ones run
 * their ADMM in independent chunks of cpd_options->chunk_sizes[m] rows, as
 * the reference runs row-separable constraints.  Anything else, and a rank
 * of 0 or above 64 (the streaming kernels' limit), returns
 * SPLATT_ERROR_BADINPUT.  Prints the driver's per-batch report lines
 * (StreamCPD.cc:509-534: local-1 every batch, global and local-10 every 100
 * batches and at the last, final-err; its "cpd" figure prints -1). */
splatt_error_type splatt_cpd_stream(char const * const filename, splatt_idx_t rank,
    splatt_idx_t const stream_mode, double const forget, splatt_cpd_opts * const cpd_options,
    splatt_global_opts const * const global_options);

/* ===== B200 extensions (no counterpart in SPLATT) ========================= */

/* Select the CUDA device (once, before other calls; default: current). */
splatt_error_type splatt_b200_init(int device);
/* The cudaStream_t every call launches on; setting it lets a caller time or
 * capture the library's work on its own stream. */
void * splatt_b200_get_stream(void);
void splatt_b200_set_stream(void * cuda_stream);
/* Text of the last CUDA error seen by the library. */
char const * splatt_b200_error_string(void);

/* Device-resident MTTKRP: `mats` and `out` are device pointers (row-major,
 * leading dimension ld / ld_out).  No host copies, no allocation.  Values
 * are double for val_type 0, float for 1; tensors must hold the same type
 * (see splatt_b200_csf_set_precision). */
splatt_error_type splatt_b200_mttkrp_device(splatt_idx_t const mode,
    splatt_idx_t const ncolumns, splatt_csf const * const tensors,
    double const * const options, void * const * mats, splatt_idx_t ld, void * out,
    splatt_idx_t ld_out, int val_type);
/* CSF trees from a COO tensor already in device memory: dinds[m] are
 * uint32 device arrays (checked < dims[m] on the device), dvals nnz values
 * of val_type (0 double, 1 float).  Scheme from options[CSF_ALLOC], as
 * splatt_csf_convert.  host_mirror = 0 skips copying fptr/fids/vals back
 * to the host struct (only nfibs is filled); the trees are then usable by
 * the device entry points only.  Free with splatt_free_csf. */
splatt_error_type splatt_b200_csf_convert_device(uint32_t nmodes, uint64_t nnz,
    uint64_t const * dims, uint32_t * const * dinds, void const * dvals, int val_type,
    splatt_csf ** tensors, double const * const options, int host_mirror);
/* Convert the device values of a CSF set to float (1) or double (0). */
splatt_error_type splatt_b200_csf_set_precision(splatt_csf * tensors,
    double const * const options, int val_type);

/* Gram matrix G = A^T A that allocates no device memory.  No counterpart in
 * SPLATT (whose mat_aTa calls BLAS dsyrk on host memory).  For callers that
 * may not call cudaMalloc / cudaFree: a process whose device memory is fully
 * partitioned between its own pools, or a plug-in whose host application
 * owns the allocator.  A (nrows x rank, leading dimension ld, double for
 * val_type 0, float for 1) and G (rank x rank doubles, upper triangle
 * written, row-major) are device pointers; the work is queued on
 * cuda_stream.  rank <= 64 (SPLATT_ERROR_BADINPUT and a stderr message
 * above that).  Per-block partial sums live in a fixed 2 MiB device array
 * that every GPU loading the library keeps until exit and that all calls on
 * a device share, keeping the last call's contents: calls that overlap on
 * the GPU race, so order them on one stream.  The first call on a device
 * looks up that array's device address; make it before any stream capture.
 * The address is cached for the device's primary context: after
 * cudaDeviceReset on a device, do not call this entry point on it again. */
splatt_error_type splatt_b200_gram_noalloc(void const * A, int val_type, uint64_t nrows,
    uint32_t rank, uint32_t ld, double * G, void * cuda_stream);

/* ---- streaming (per-slice) handle --------------------------------------- */
typedef struct splatt_b200_stream splatt_b200_stream;

/* Precision of a stream's per-slice update. */
typedef enum {
  SPLATT_B200_FP64 = 0,       /* everything in FP64 (the plain path) */
  SPLATT_B200_FP32 = 1        /* FP32 factors + MTTKRP, 3xTF32 Grams, FP64
                                 Cholesky/solve and fit accumulation */
} splatt_b200_precision;

/* Execution strategy of the per-slice update. */
typedef enum {
  SPLATT_B200_PLAIN = 0,      /* one kernel per step, host-driven loops */
  SPLATT_B200_FUSED = 1       /* persistent fused slice kernel */
} splatt_b200_exec;

/* A streaming CPD of an (nmodes)-mode tensor whose mode `stream_mode` is
 * time, mirroring StreamCPD::compute (src/cpd/stream/StreamCPD.cc:311-571).
 * `max_dims[m]` bounds the rows of each non-streamed factor (device state is
 * sized once); the random stream for new rows is glibc rand() as in SPLATT
 * (seed with srand before the first slice). */
splatt_b200_stream * splatt_b200_stream_alloc(splatt_idx_t nmodes,
    splatt_idx_t stream_mode, splatt_idx_t const * max_dims, splatt_idx_t rank,
    double forget, double reg, splatt_idx_t max_iterations,
    splatt_b200_precision precision, splatt_b200_exec exec);
void splatt_b200_stream_free(splatt_b200_stream * s);
/* Process one time slice given as host COO (indices already relabelled so
 * that each non-streamed mode's new indices appear in first-use order, as
 * SPLATT's ParserSimple does; the time index is ignored).  Writes the new
 * time row to time_row (rank values; may be NULL) and returns the outer
 * iterations taken (0 on error; see splatt_b200_stream_status). */
splatt_idx_t splatt_b200_stream_push(splatt_b200_stream * s, splatt_idx_t nnz,
    splatt_idx_t ** inds, splatt_val_t const * vals, splatt_val_t * time_row);
/* As above with the slice already on the device (uint32 indices per mode,
 * values of the stream's precision).  Asynchronous: nothing is read back. */
splatt_error_type splatt_b200_stream_push_device(splatt_b200_stream * s,
    splatt_idx_t nnz, uint32_t * const * dinds, void const * dvals,
    splatt_idx_t const * slice_dims);
splatt_error_type splatt_b200_stream_status(splatt_b200_stream const * s);
/* The prox of non-streamed mode `mode`'s ADMM: max-column-norm (the
 * default, maxcolnorm.c:32-62), the non-negative max-column-norm
 * (maxcolnorm-nonneg.c:32-62), lasso (lasso.c:32-55: soft threshold at
 * multiplier / rho), each row onto the probability simplex (simplex.cc:
 * 34-66), NTF-L1 (nonneg_lasso.c:30-45: v > multiplier / rho ?
 * v - multiplier / rho : 0) or NTF-Frobenius (nonneg_frob.c:31-49:
 * max(v * rho / (multiplier + rho), 0)).  The last four are row-separable,
 * and their ADMM runs in independent chunks of chunk_rows rows, 0 = 50
 * (src/cpd/admm.c:352-395).  Takes effect from the next slice. */
typedef enum {
  SPLATT_B200_PROX_MAXCOLNORM = 0,
  SPLATT_B200_PROX_MAXCOLNORM_NONNEG = 1,
  SPLATT_B200_PROX_LASSO = 2,
  SPLATT_B200_PROX_ROWSIMP = 3,
  SPLATT_B200_PROX_NTF_LASSO = 4,
  SPLATT_B200_PROX_NTF_FROB = 5,
  SPLATT_B200_PROX_COLSIMP = 6   /* each column onto the probability simplex
                                    (simplex.cc:113-150; single-chunk ADMM) */
} splatt_b200_prox;
splatt_error_type splatt_b200_stream_set_prox(splatt_b200_stream * s, splatt_idx_t mode,
    splatt_b200_prox kind, double multiplier, splatt_idx_t chunk_rows);
/* Give the stream its own generator for new factor rows (rand_r seeded with
 * `seed`) instead of the process-wide rand() SPLATT uses, so its result does
 * not depend on which other streams share the process (serving, batches). */
void splatt_b200_stream_seed(splatt_b200_stream * s, unsigned seed);
/* Device memory held by the stream's resident state. */
size_t splatt_b200_stream_bytes(splatt_b200_stream const * s);
/* Copy the current factors to host: factors[m] gets rows x rank values
 * (non-streamed modes), rows[m] the row counts, time row for stream_mode. */
splatt_error_type splatt_b200_stream_factors(splatt_b200_stream * s,
    splatt_val_t ** factors, splatt_idx_t * rows);
/* Per-slice error^2 of the latest slice (SPLATT's "local-1" figure,
 * src/cpd/stream/StreamCPD.cc:77-86) computed on the device in FP64. */
double splatt_b200_stream_local_errsq(splatt_b200_stream * s);
/* Error^2 of the current model on the last min(k, slices so far) slices
 * (StreamCPD::compute_errorsq(k), StreamCPD.cc:77-86: the current factors,
 * the time rows of those slices; the driver's "global" figure for k = all
 * slices, "local-10" for k = 10): (||X||^2 + ||Z||^2 - 2<X, Z>) / ||X||^2.
 * The window's nonzeros are given on the device (nnz of them, uint32
 * indices per mode, the streamed mode's holding absolute slice numbers,
 * FP64 values), e.g. a range of a prepared stream.  FP64 arithmetic.
 * Returns -1 on failure. */
double splatt_b200_stream_window_errsq(splatt_b200_stream * s, splatt_idx_t nnz,
    uint32_t * const * dinds, double const * dvals, splatt_idx_t k);
/* Outer iterations of the last slice; ADMM inner iterations of the last
 * slice for a non-streamed mode (summed over its outer iterations); current
 * rows of a factor (for the streamed mode: slices processed). */
splatt_idx_t splatt_b200_stream_last_outer(splatt_b200_stream const * s);
/* Wait for the stream's queued work and refresh the iteration counts above
 * (push_device does not wait); reports a device-side error if one occurred. */
splatt_error_type splatt_b200_stream_sync(splatt_b200_stream * s);
splatt_idx_t splatt_b200_stream_last_inner(splatt_b200_stream const * s, splatt_idx_t mode);
splatt_idx_t splatt_b200_stream_rows(splatt_b200_stream const * s, splatt_idx_t mode);

/* ---- many streams: batched slice updates (no counterpart in SPLATT) ----- */
typedef struct splatt_b200_batch splatt_b200_batch;

/* A batch holds up to max_slices slices of streams of one precision (rank
 * <= max_rank <= 64); several slices of one stream may be staged, they form
 * a chain and run in the order added.  One cooperative launch updates them
 * all: fixed groups of blocks claim chains dynamically (the chain with the
 * most slices left first), so a slow slice holds only its own group.  The
 * launch is replayed from a CUDA graph after the first call. */
splatt_b200_batch * splatt_b200_batch_alloc(splatt_idx_t max_slices,
    splatt_b200_precision precision, splatt_idx_t max_rank);
void splatt_b200_batch_free(splatt_b200_batch * b);
/* Stage stream s's next slice (device COO as for stream_push_device; the
 * arrays must stay valid until the batch has been synced).  FUSED streams
 * only. */
splatt_error_type splatt_b200_batch_add(splatt_b200_batch * b, splatt_b200_stream * s,
    splatt_idx_t nnz, uint32_t * const * dinds, void const * dvals,
    splatt_idx_t const * slice_dims);
/* Launch the staged slices (asynchronous), then wait for them. */
splatt_error_type splatt_b200_batch_run(splatt_b200_batch * b);
splatt_error_type splatt_b200_batch_sync(splatt_b200_batch * b);
/* Blocks per group (0: automatic, max(1, blocks / streams in the batch)). */
void splatt_b200_batch_set_group(splatt_b200_batch * b, int blocks_per_group);
/* Blocks per group of the last launch. */
int splatt_b200_batch_last_group(splatt_b200_batch const * b);
/* Multiplier of the automatic group size (the serving loop's autotuner sets
 * it per batch; default 1). */
void splatt_b200_batch_set_factor(splatt_b200_batch * b, int factor);
/* 1 when launches replay a captured CUDA graph, 0 when capture was not
 * available (direct launches), -1 before the first run. */
int splatt_b200_batch_graph_used(splatt_b200_batch const * b);
int splatt_b200_batch_blocks(splatt_b200_batch const * b);

/* ---- serving loop (no counterpart in SPLATT) ---------------------------- */
typedef struct splatt_b200_server splatt_b200_server;

/* Streams are admitted while their resident state fits hbm_budget_bytes;
 * a batch holds up to max_batch slices (several per stream when they have
 * arrived). */
splatt_b200_server * splatt_b200_server_alloc(size_t hbm_budget_bytes,
    splatt_b200_precision precision, splatt_idx_t max_batch, splatt_idx_t max_rank);
void splatt_b200_server_free(splatt_b200_server * v);
/* Register a stream (StreamCPD semantics, its own row generator seeded
 * with `seed`); returns its id, admitted when memory allows. */
int splatt_b200_server_open(splatt_b200_server * v, splatt_idx_t nmodes,
    splatt_idx_t stream_mode, splatt_idx_t const * max_dims, splatt_idx_t rank, double forget,
    double reg, splatt_idx_t max_iterations, unsigned seed);
/* Release a stream's device state (not while one of its slices runs). */
splatt_error_type splatt_b200_server_close(splatt_b200_server * v, int id);
int splatt_b200_server_admitted(splatt_b200_server const * v, int id);
/* Queue a slice (host COO, first-use relabelled indices) that arrived at
 * `arrival` on the caller's clock (seconds). */
splatt_error_type splatt_b200_server_submit(splatt_b200_server * v, int id, splatt_idx_t nnz,
    splatt_idx_t ** inds, splatt_val_t const * vals, double arrival);
/* Non-blocking scheduling step at time `now`: completes the batch in flight
 * if it has finished, admits waiting streams, launches the next batch from
 * the queued slices with arrival <= now.  Returns the slices completed. */
splatt_idx_t splatt_b200_server_poll(splatt_b200_server * v, double now);
/* Run every queued slice to completion. */
splatt_error_type splatt_b200_server_drain(splatt_b200_server * v, double now);
/* Slice latency percentiles (completion poll - arrival), counts. */
splatt_error_type splatt_b200_server_stats(splatt_b200_server const * v, double * p50,
    double * p99, splatt_idx_t * completed, splatt_idx_t * batches);
/* Forget the latencies and batch count recorded so far. */
void splatt_b200_server_reset_stats(splatt_b200_server * v);
splatt_b200_stream * splatt_b200_server_stream(splatt_b200_server * v, int id);
size_t splatt_b200_server_used(splatt_b200_server const * v);
/* Slices of the launched batch that the GPU is still running (0 when no
 * batch is launched or the GPU has finished it; a poll then completes it). */
splatt_idx_t splatt_b200_server_inflight(splatt_b200_server * v);

#ifdef __cplusplus
}
#endif

#endif
