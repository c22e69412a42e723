/*
 * mttkrp.c -- splatt_mttkrp and its workspace (include/splatt/api_kernels.h,
 * src/mttkrp.c:1287-1343, 1775-1945).
 *
 * splatt_mttkrp keeps SPLATT's contract: host row-major factors in, the
 * output matrix zeroed and overwritten.  The tree serving `mode` and the
 * traversal depth follow mttkrp_csf (root / internal / leaf by the mode's
 * level in that tree); the traversal itself is one device kernel.
 */
#include "sb_host.h"

splatt_mttkrp_ws * splatt_mttkrp_alloc_ws(splatt_csf const * const tensors,
    splatt_idx_t const ncolumns, double const * const opts)
{
  (void) ncolumns;
  splatt_mttkrp_ws * ws = calloc(1, sizeof(*ws));
  idx_t const N = tensors->nmodes;
  ws->num_csf = sb_csf_count(tensors, opts);
  ws->num_threads = 1;
  for(idx_t m = 0; m < N; ++m) {
    ws->mode_csf_map[m] = sb_mode_csf(tensors, ws->num_csf, m);
    /* src/mttkrp.c:221-236: one host thread never privatises; the device
     * resolves output conflicts with atomics instead */
    ws->is_privatized[m] = false;
  }
  ws->privatize_buffer = NULL;
  return ws;
}

void splatt_mttkrp_free_ws(splatt_mttkrp_ws * const ws) { free(ws); }

/* device MTTKRP on tree `t` for `mode` with factors by mode */
static int p_mttkrp_dev(splatt_csf const * t, idx_t mode, idx_t R, void * const * mats,
    idx_t ld, void * out, idx_t ld_out, int vt)
{
  if(!t->dev) { return SB_EINPUT; }
  void * bylevel[SB_MAX_NMODES];
  for(idx_t l = 0; l < t->nmodes; ++l) { bylevel[l] = mats[t->dim_perm[l]]; }
  return sb_tree_mttkrp(t, (uint32_t) t->dim_iperm[mode], (uint32_t) R, bylevel,
      (uint32_t) ld, out, (uint32_t) ld_out, vt);
}

int splatt_mttkrp(splatt_idx_t const mode, splatt_idx_t const ncolumns,
    splatt_csf const * const tensors, splatt_val_t ** matrices, splatt_val_t * const matout,
    double const * const options)
{
  if(!tensors || !matrices || !matout || mode >= tensors->nmodes || ncolumns == 0) {
    return SPLATT_ERROR_BADINPUT;
  }
  int rc = sb_ensure_init();
  if(rc) { return sb_err(rc); }
  idx_t const N = tensors->nmodes;
  idx_t const ncsf = sb_csf_count(tensors, options);
  splatt_csf const * t = tensors + sb_mode_csf(tensors, ncsf, mode);
  void * dm[SB_MAX_NMODES] = {0};
  void * dout = NULL;
  size_t const vb = sizeof(val_t);
  for(idx_t m = 0; m < N && rc == SB_OK; ++m) {
    if(m == mode) { continue; }
    rc = sb_malloc(&dm[m], tensors->dims[m] * ncolumns * vb);
    if(rc == SB_OK) { rc = sb_h2d(dm[m], matrices[m], tensors->dims[m] * ncolumns * vb); }
  }
  if(rc == SB_OK) { rc = sb_malloc(&dout, tensors->dims[mode] * ncolumns * vb); }
  if(rc == SB_OK) { rc = p_mttkrp_dev(t, mode, ncolumns, dm, ncolumns, dout, ncolumns, SB_VT); }
  if(rc == SB_OK) { rc = sb_d2h(matout, dout, tensors->dims[mode] * ncolumns * vb); }
  for(idx_t m = 0; m < N; ++m) { sb_free(dm[m]); }
  sb_free(dout);
  return rc == SB_OK ? SPLATT_SUCCESS : sb_err(rc);
}

splatt_error_type splatt_b200_mttkrp_device(splatt_idx_t const mode,
    splatt_idx_t const ncolumns, splatt_csf const * const tensors,
    double const * const options, void * const * mats, splatt_idx_t ld, void * out,
    splatt_idx_t ld_out, int val_type)
{
  if(!tensors || mode >= tensors->nmodes || ncolumns == 0) { return SPLATT_ERROR_BADINPUT; }
  idx_t const ncsf = sb_csf_count(tensors, options);
  splatt_csf const * t = tensors + sb_mode_csf(tensors, ncsf, mode);
  return sb_err(p_mttkrp_dev(t, mode, ncolumns, mats, ld, out, ld_out, val_type));
}
