/*
 * sb_host.h -- internal declarations shared by the C host files.
 */
#ifndef SPLATT_B200_HOST_H
#define SPLATT_B200_HOST_H

#include "../../../include/splatt_b200.h"
#include "../kernels/kapi.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

typedef splatt_idx_t idx_t;
typedef splatt_val_t val_t;

#define SB_VT ((SPLATT_VAL_TYPEWIDTH == 32) ? SB_F32 : SB_F64)

/* map a kapi status to a SPLATT error code */
static inline splatt_error_type sb_err(int rc)
{
  switch(rc) {
  case SB_OK: return SPLATT_SUCCESS;
  case SB_ENOMEM: return SPLATT_ERROR_NOMEMORY;
  case SB_EINPUT: return SPLATT_ERROR_BADINPUT;
  default: return SPLATT_ERROR_DEVICE;
  }
}

/* lazily initialise the device (current device) */
int sb_ensure_init(void);

/* mode orderings (src/csf.c:93-218, 608-651) */
void sb_order_small(idx_t const * dims, idx_t nmodes, idx_t * perm);
void sb_order_minusone(idx_t const * dims, idx_t nmodes, idx_t special, idx_t * perm);

/* number of CSF trees for an allocation scheme */
idx_t sb_csf_count(splatt_csf const * tensors, double const * opts);

/* which tree serves MTTKRP `mode` (src/mttkrp.c:1849-1880) */
idx_t sb_mode_csf(splatt_csf const * tensors, idx_t ncsf, idx_t mode);
/* MTTKRP of one (possibly dense-tiled) tree into out (zeroed first) */
int sb_tree_mttkrp(splatt_csf const * t, uint32_t out_level, uint32_t R,
    void * const * mats_by_level, uint32_t ld, void * out, uint32_t ld_out, int vt);
/* sum of squared nonzero values of one tree */
int sb_tree_frobsq(splatt_csf const * t, double * out);
/* device COO from host arrays: uint32 indices (checked < dims), val_t values */
int sb_upload_coo(idx_t nmodes, idx_t nnz, idx_t const * dims, idx_t * const * inds,
    val_t const * vals, uint32_t ** dind, void ** dval);

/* 1 for a constraint registered by splatt_register_ntf_frob (its description
 * is the same as splatt_register_ntf_lasso's) */
int sb_con_is_ntf_frob(splatt_cpd_constraint const * c);

/* glibc-rand factor fill (src/util.c:15-40) */
void sb_fill_rand(val_t * v, idx_t n);

/* COO readers (src/io.c): returns NULL on failure */
splatt_coord * sb_read_tensor(char const * fname);
/* The same file read onto the device (uint32 indices, val_t values, both
 * allocated by the call; SB_* codes): text parsed by the device, binary
 * widths converted and ranges checked there. */
int sb_read_tensor_device(char const * fname, idx_t * nmodes, idx_t * nnz, idx_t * dims,
    uint32_t ** dinds, void ** dvals);
/* The mode count of a .tns / .bin file from its first data line or header
 * (no device work); SB_EINPUT for a missing file or a bad count. */
int sb_file_modes(char const * fname, idx_t * nmodes);
/* drop empty slices, renumbering kept indices (src/sptensor.c:190-252);
 * returns the slices removed, or (idx_t) -1 when a host allocation failed */
idx_t sb_remove_empty(splatt_coord * tt);

#endif
