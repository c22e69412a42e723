/*
 * kapi.h -- the thin C-ABI between the C host code and the sm_100a kernels.
 *
 * Plain C: pointers, sizes and status codes only.  Every function is
 * implemented in a .cu file of csrc/kernels and launches on the library's
 * current CUDA stream (sb_get_stream) unless a stream is passed explicitly.
 * Device-side index arrays are uint32 (dimensions and nonzero counts must stay
 * below 2^32 - 1); values are float (SB_F32) or double (SB_F64).
 *
 * Return codes: 0 = success, SB_ENOMEM = device allocation failed,
 * SB_EDEVICE = any other CUDA error, SB_EINPUT = invalid arguments.
 */
#ifndef SPLATT_B200_KAPI_H
#define SPLATT_B200_KAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SB_MAX_NMODES 8
#define SB_F64 0
#define SB_F32 1

#define SB_OK 0
#define SB_ENOMEM 1
#define SB_EDEVICE 2
#define SB_EINPUT 3

/* ---- device CSF (one tree) --------------------------------------------- */
typedef struct {
  uint32_t nmodes;
  uint64_t nnz;
  uint64_t dims[SB_MAX_NMODES];
  uint32_t dim_perm[SB_MAX_NMODES];   /* level -> mode */
  uint64_t nfibs[SB_MAX_NMODES];
  uint32_t * fptr[SB_MAX_NMODES];     /* levels 0..nmodes-2, nfibs[l]+1 */
  uint32_t * fids[SB_MAX_NMODES];     /* levels 0..nmodes-1 (root kept) */
  void * vals;                        /* nnz values, val_type */
  int val_type;
} sb_dcsf;

/* ---- runtime ----------------------------------------------------------- */
int sb_init(int device);
void * sb_get_stream(void);
void sb_set_stream(void * stream);
int sb_sync(void);
int sb_stream_sync(void * stream);
int sb_malloc(void ** p, size_t bytes);
int sb_free(void * p);
int sb_memset(void * p, int v, size_t bytes);
int sb_h2d(void * dst, void const * src, size_t bytes);
int sb_d2h(void * dst, void const * src, size_t bytes);
int sb_d2d(void * dst, void const * src, size_t bytes);
/* capture the calls made between begin and end (on the library stream) into
 * a CUDA graph; end returns an error and no graph when the capture failed */
int sb_capture_begin(void);
int sb_capture_end(void ** exec);
int sb_graph_launch(void * graph_exec);
void sb_graph_destroy(void * graph_exec);
int sb_host_alloc(void ** p, size_t bytes);    /* pinned host memory */
void sb_host_free(void * p);
int sb_last_error(void);
char const * sb_error_string(void);
size_t sb_mem_free(void);
int sb_device_count(void);

/* ---- sorting / scan ---------------------------------------------------- */
/* out[i] = sum_{k<i} in[k]; returns the total in *total (may be NULL). */
int sb_exclusive_scan_u32(uint32_t const * in, uint32_t * out, uint64_t n,
    uint64_t * total);
/* Stable LSD sort of (keys, vals) by the low `bits` bits of keys.  Buffers are
 * ping-ponged with the *_alt arrays; on return *result_in_alt tells where the
 * sorted data is. */
int sb_radix_sort_pairs(uint32_t * keys, uint32_t * vals, uint32_t * keys_alt,
    uint32_t * vals_alt, uint64_t n, int bits, int * result_in_alt);

/* ---- CSF build ---------------------------------------------------------- */
/* Build a device CSF from device COO (inds[m]: uint32 per mode, vals of
 * val_type) under the level->mode order dim_perm.  All output arrays are
 * allocated by the call and owned by `out`.  Inputs are not modified. */
int sb_csf_build(uint32_t nmodes, uint64_t nnz, uint64_t const * dims,
    uint32_t * const * inds, void const * vals, int val_type,
    uint32_t const * dim_perm, sb_dcsf * out);
void sb_csf_release(sb_dcsf * c);
/* Dense tiling (src/tile.c:260-340): nonzeros grouped by tile id, tile id =
 * sum over modes of min(ind / tsize[m], tdim[m] - 1) times the product of
 * the later modes' tdim (mode 0 slowest); ntiles = prod tdim <= 2^24.
 * inds_out[m] / vals_out hold nnz entries; counts (host) gets ntiles. */
int sb_tile_partition(uint32_t nmodes, uint64_t nnz, uint32_t * const * inds,
    void const * vals, int val_type, uint64_t const * tsize, uint32_t const * tdim,
    uint64_t ntiles, uint32_t * const * inds_out, void * vals_out, uint64_t * counts);
/* Narrow host-width device indices to uint32, checking idx < dim; returns
 * SB_EINPUT if any index is out of range. */
int sb_narrow_u64(uint64_t const * src, uint32_t * dst, uint64_t n,
    uint64_t dim);
int sb_check_u32(uint32_t const * src, uint64_t n, uint64_t dim);
/* Sum of squares of the values (double accumulation). */
int sb_frobsq(void const * vals, int val_type, uint64_t n, double * out);
int sb_convert_vals(void const * src, int src_type, void * dst, int dst_type,
    uint64_t n);

/* ---- streaming ingest ------------------------------------------------------ */
/* ParserSimple's preparation on the device (src/cpd/stream/ParserSimple.cc:
 * 13-149): out_inds / out_vals (nnz each) = the nonzeros ordered by (sm, then
 * the following modes cyclically), every mode but sm relabelled by first
 * appearance; iperm[m] (dims[m] entries, m != sm) = original index of each
 * label, nlabels[m] (host) = labels used; offs (host, dims[sm] + 1) = slice
 * boundaries; seen (host, row m of dims[sm] entries) = labels of mode m seen
 * up to the end of each slice.  Inputs are not modified. */
int sb_stream_prepare(uint32_t nmodes, uint64_t nnz, uint64_t const * dims,
    uint32_t * const * inds, void const * vals, int val_type, uint32_t stream_mode,
    uint32_t * const * out_inds, void * out_vals, uint32_t * const * iperm,
    uint64_t * nlabels, uint64_t * offs, uint64_t * seen);

/* ---- file ingest ------------------------------------------------------- */
/* Parse a text tensor (the host bytes hbuf[0, nbytes) of a .tns file with
 * nmodes indices per line) on the device: inds[m] (uint32, 0-based, nnz
 * each) and vals (FP64) are allocated by the call; dims (host) gets each
 * mode's size; *nfallback the lines the device could not parse exactly,
 * re-read on the host. */
int sb_parse_text(char const * hbuf, uint64_t nbytes, uint32_t nmodes, uint32_t ** inds,
    double ** vals, uint64_t * nnz_out, uint64_t * dims, uint64_t * nfallback);
/* tt_remove_empty on device COO: every mode's used indices renumbered in
 * increasing order, dims (host) shrunk; indmap[m] (device, may be NULL)
 * new -> old for the modes that shrank (NULL for the others). */
int sb_remove_empty_device(uint32_t nmodes, uint64_t nnz, uint64_t * dims,
    uint32_t * const * inds, uint32_t ** indmap, uint64_t * removed);

/* ---- MTTKRP -------------------------------------------------------------- */
/* out[dims[mode]][ld_out] = MTTKRP of the CSF for output level `out_level`.
 * mats_by_level[l] is the factor of mode dim_perm[l] (row-major, leading
 * dimension ld).  Columns [0, R).  `out` is overwritten (zeroed first). */
int sb_mttkrp_csf(sb_dcsf const * c, uint32_t out_level, uint32_t R,
    void * const * mats_by_level, uint32_t ld, void * out, uint32_t ld_out,
    int val_type);
/* The same, adding into `out` (zeroed first only when `zero`): the tiles of
 * a dense-tiled tree are summed one after another. */
int sb_mttkrp_csf_acc(sb_dcsf const * c, uint32_t out_level, uint32_t R,
    void * const * mats_by_level, uint32_t ld, void * out, uint32_t ld_out,
    int val_type, int zero);
/* The CSF MTTKRP autotuner (on by default): 0 always uses the heuristic
 * launch shape.  sb_mttkrp_tune_table copies up to max_entries tuned
 * buckets, 8 ints each (value type, levels, output kind 0 root / 1
 * internal / 2 leaf, log2 rank, log4 nnz, V, G, chunk), and returns how
 * many there are. */
void sb_mttkrp_autotune(int on);
int sb_mttkrp_tune_table(int * out, int max_entries);
/* COO MTTKRP (device arrays): out[inds[mode][n]] += v_n * prod_{m!=mode}
 * mats[m][inds[m][n]].  out is zeroed first (rows out_rows). */
int sb_mttkrp_coo(uint32_t nmodes, uint64_t nnz, uint32_t * const * inds,
    void const * vals, uint32_t mode, uint32_t R, void * const * mats,
    uint32_t ld, void * out, uint64_t out_rows, int val_type);

/* ---- dense -------------------------------------------------------------- */
/* G[R][R] (upper triangle, row-major, double) = A^T A for A[I][ld] of
 * val_type; precision: 0 = FP64 FMA, 1 = 3xTF32 tensor-core split products
 * (val_type SB_F32 only). */
int sb_gram(void const * A, int val_type, uint64_t I, uint32_t R, uint32_t ld,
    double * G, int precision);
/* G (R x R) = A^T A of an FP32 A on the tensor cores (tcgen05 kind::tf32,
 * split hi/lo products, FP32 accumulation per <= 4096 rows, FP64 across);
 * R <= 64 */
int sb_gram_tc(float const * A, uint64_t I, uint32_t R, uint32_t ld, double * G);
#define SB_GRAM_TF32X3 1   /* sb_gram precision: split TF32 tensor-core products */
/* Fused: G = Hadamard_{m != skip} grams[m] (upper), + diag_add (+ trace/R
 * when add_trace_rho), Cholesky in FP64.  rho_out (device, may be NULL)
 * receives the rho used.  status (device int) gets the failing pivot + 1. */
int sb_form_gram_chol(double const * const * grams, uint32_t ngrams,
    uint32_t skip, uint32_t R, double diag_add, int add_trace_rho,
    double * L, double * rho_out, int * status);
/* B[I][ld] <- rows solved against L (forward + backward), FP64 math. */
int sb_chol_solve(double const * L, uint32_t R, void * B, int val_type,
    uint64_t I, uint32_t ld);
/* Column 2-norms -> lambda (device double[R]) and divide A by them. */
int sb_normalize(void * A, int val_type, uint64_t I, uint32_t R, uint32_t ld,
    double * lambda);
/* fit pieces: inner = sum_r lambda[r] * sum_i A[i][r] * M[i][r] */
int sb_inner(void const * A, void const * M, int val_type, uint64_t I,
    uint32_t R, uint32_t ld, double const * lambda, double * out);

/* ---- bounded waits ----------------------------------------------------- */
/* Deadline (ns) of every grid-barrier wait of the streaming kernels; 0
 * restores the default 2 s.  An expired wait sets the launch's error word,
 * every block returns, and the host call reports SPLATT_ERROR_DEVICE. */
int sb_set_wait_deadline_ns(uint64_t ns);

/* ---- events (timing) ------------------------------------------------- */
int sb_event_create(void ** ev);
int sb_event_record(void * ev, void * stream);
int sb_event_elapsed_ms(void * a, void * b, float * ms);
int sb_event_destroy(void * ev);
int sb_event_sync(void * ev);

#ifdef __cplusplus
}
#endif
#endif
