/*
 * csf.c -- CSF allocation / conversion / release (host side of the build).
 *
 * Mirrors csf_alloc (src/csf.c:695-739) and p_mk_csf (527-558): ONEMODE =
 * one tree rooted at the shortest mode (CSF_SORTED_SMALLFIRST); TWOMODE =
 * that tree plus one rooted at its leaf mode (CSF_SORTED_MINUSONE); ALLMODE =
 * one MINUSONE tree per mode.  The trees are built on the device by
 * sb_csf_build; the host struct mirrors SPLATT's (fptr/fids/vals copied back,
 * root fids NULL for an untiled tree as SPLATT leaves it) and `dev` holds the
 * device arrays used by every kernel.
 */
#include "sb_host.h"

idx_t sb_csf_count(splatt_csf const * tensors, double const * opts)
{
  switch((int) opts[SPLATT_OPTION_CSF_ALLOC]) {
  case SPLATT_CSF_ONEMODE: return 1;
  case SPLATT_CSF_TWOMODE: return 2;
  default: return tensors[0].nmodes;
  }
}

idx_t sb_mode_csf(splatt_csf const * tensors, idx_t ncsf, idx_t mode)
{
  idx_t const N = tensors[0].nmodes;
  if(ncsf == 1) { return 0; }
  if(ncsf == 2) { return tensors[0].dim_iperm[mode] == N - 1 ? 1 : 0; }
  return mode;
}

/* copy a device uint32 array to a host idx_t array */
static int p_d2h_idx(idx_t * dst, uint32_t const * src, idx_t n)
{
  if(n == 0) { return SB_OK; }
#if SPLATT_IDX_TYPEWIDTH == 32
  return sb_d2h(dst, src, n * sizeof(uint32_t));
#else
  uint32_t * tmp = malloc(n * sizeof(uint32_t));
  int rc = sb_d2h(tmp, src, n * sizeof(uint32_t));
  for(idx_t i = 0; rc == SB_OK && i < n; ++i) { dst[i] = tmp[i]; }
  free(tmp);
  return rc;
#endif
}

/* device COO (uint32 indices + values of val_t) from host arrays */
int sb_upload_coo(idx_t nmodes, idx_t nnz, idx_t const * dims, idx_t * const * inds,
    val_t const * vals, uint32_t ** dind, void ** dval)
{
  int rc = SB_OK;
  for(idx_t m = 0; m < nmodes; ++m) { dind[m] = NULL; }
  *dval = NULL;
  for(idx_t m = 0; m < nmodes && rc == SB_OK; ++m) {
    if(dims[m] >= 0xffffffffull) { return SB_EINPUT; }
    rc = sb_malloc((void **) &dind[m], nnz * sizeof(uint32_t));
    if(rc) { break; }
#if SPLATT_IDX_TYPEWIDTH == 32
    rc = sb_h2d(dind[m], inds[m], nnz * sizeof(uint32_t));
    if(rc == SB_OK) { rc = sb_check_u32(dind[m], nnz, dims[m]); }
#else
    uint64_t * wide = NULL;
    rc = sb_malloc((void **) &wide, nnz * sizeof(uint64_t));
    if(rc == SB_OK) { rc = sb_h2d(wide, inds[m], nnz * sizeof(uint64_t)); }
    if(rc == SB_OK) { rc = sb_narrow_u64(wide, dind[m], nnz, dims[m]); }
    sb_free(wide);
#endif
  }
  if(rc == SB_OK) { rc = sb_malloc(dval, nnz * sizeof(val_t)); }
  if(rc == SB_OK) { rc = sb_h2d(*dval, vals, nnz * sizeof(val_t)); }
  if(rc) {
    for(idx_t m = 0; m < nmodes; ++m) { sb_free(dind[m]); dind[m] = NULL; }
    sb_free(*dval);
    *dval = NULL;
  }
  return rc;
}

static int p_mk_csf_typed(splatt_csf * ct, idx_t nmodes, idx_t nnz, idx_t const * dims,
    uint32_t * const * dind, void const * dval, idx_t const * perm, int val_type, int mirror,
    double const * tile_opts);

/* build tree `ct` from the uploaded COO with level order `perm` */
static int p_mk_csf(splatt_csf * ct, idx_t nmodes, idx_t nnz, idx_t const * dims,
    uint32_t * const * dind, void const * dval, idx_t const * perm, double const * tile_opts)
{
  return p_mk_csf_typed(ct, nmodes, nnz, dims, dind, dval, perm, SB_VT, 1, tile_opts);
}

/* dense-tile geometry of one tree (src/csf.c:433-451): the modes at the
 * bottom SPLATT_OPTION_TILELEVEL levels get SPLATT_OPTION_NTHREADS index
 * ranges of dims / NTHREADS (at least 1) each */
static idx_t p_tile_geom(splatt_csf * ct, double const * opts, uint64_t * tsize,
    uint32_t * tdim)
{
  idx_t const N = ct->nmodes;
  idx_t ntiled = (idx_t) opts[SPLATT_OPTION_TILELEVEL];
  if(ntiled > N) { ntiled = N; }
  idx_t const T = opts[SPLATT_OPTION_NTHREADS] >= 1 ? (idx_t) opts[SPLATT_OPTION_NTHREADS] : 1;
  ct->ntiled_modes = ntiled;
  idx_t ntiles = 1;
  for(idx_t m = 0; m < N; ++m) {
    ct->tile_dims[m] = ct->dim_iperm[m] >= N - ntiled ? T : 1;
    tdim[m] = (uint32_t) ct->tile_dims[m];
    tsize[m] = ct->dims[m] / ct->tile_dims[m] > 0 ? ct->dims[m] / ct->tile_dims[m] : 1;
    ntiles *= ct->tile_dims[m];
  }
  return ntiles;
}

/* host mirror of one tile (SPLATT keeps root ids only when the tree has
 * more than one tile, src/csf.c:258-264; an empty tile keeps a {0, 0} root
 * pointer and nothing else, src/csf.c:466-479) */
static int p_mirror(csf_sparsity * pt, sb_dcsf const * d, idx_t nmodes, int val_type,
    int root_ids)
{
  int rc = SB_OK;
  for(idx_t l = 0; l < nmodes; ++l) { pt->nfibs[l] = d->nfibs[l]; }
  if(d->nnz == 0) {
    pt->fptr[0] = calloc(2, sizeof(idx_t));
    return SB_OK;
  }
  for(idx_t l = 0; l + 1 < nmodes && rc == SB_OK; ++l) {
    pt->fptr[l] = malloc((pt->nfibs[l] + 1) * sizeof(idx_t));
    rc = p_d2h_idx(pt->fptr[l], d->fptr[l], pt->nfibs[l] + 1);
    if((l > 0 || root_ids) && rc == SB_OK) {
      pt->fids[l] = malloc((pt->nfibs[l] ? pt->nfibs[l] : 1) * sizeof(idx_t));
      rc = p_d2h_idx(pt->fids[l], d->fids[l], pt->nfibs[l]);
    }
  }
  if(rc == SB_OK) {
    pt->fids[nmodes-1] = malloc(d->nnz * sizeof(idx_t));
    rc = p_d2h_idx(pt->fids[nmodes-1], d->fids[nmodes-1], d->nnz);
  }
  if(rc == SB_OK && val_type == SB_VT) {
    pt->vals = malloc(d->nnz * sizeof(val_t));
    rc = sb_d2h(pt->vals, d->vals, d->nnz * sizeof(val_t));
  }
  return rc;
}

/* One tree; with tile_opts (SPLATT_DENSETILE) one device CSF per tile, the
 * nonzeros bucketed by tile on the device and every tile built like an
 * untiled tree over its own nonzeros (src/csf.c:427-501). */
static int p_mk_csf_typed(splatt_csf * ct, idx_t nmodes, idx_t nnz, idx_t const * dims,
    uint32_t * const * dind, void const * dval, idx_t const * perm, int val_type, int mirror,
    double const * tile_opts)
{
  memset(ct, 0, sizeof(*ct));
  ct->nnz = nnz;
  ct->nmodes = nmodes;
  uint32_t p32[SB_MAX_NMODES];
  uint64_t d64[SB_MAX_NMODES];
  for(idx_t m = 0; m < nmodes; ++m) {
    ct->dims[m] = dims[m];
    ct->dim_perm[m] = perm[m];
    p32[m] = (uint32_t) perm[m];
    d64[m] = dims[m];
    ct->tile_dims[m] = 1;
  }
  for(idx_t l = 0; l < nmodes; ++l) { ct->dim_iperm[ct->dim_perm[l]] = l; }
  ct->which_tile = SPLATT_NOTILE;
  ct->ntiles = 1;
  ct->ntiled_modes = 0;
  uint64_t tsize[SB_MAX_NMODES];
  uint32_t tdim[SB_MAX_NMODES];
  if(tile_opts) {
    ct->which_tile = SPLATT_DENSETILE;
    ct->ntiles = p_tile_geom(ct, tile_opts, tsize, tdim);
  }
  idx_t const nt = ct->ntiles;
  if(nt > (1u << 24)) { return SB_EINPUT; }
  sb_dcsf * d = calloc(nt, sizeof(*d));
  ct->dev = d;
  ct->pt = calloc(nt, sizeof(csf_sparsity));
  int rc = SB_OK;
  if(nt == 1) {
    rc = sb_csf_build((uint32_t) nmodes, nnz, d64, (uint32_t * const *) dind, dval, val_type,
        p32, d);
  } else {
    size_t const vb = val_type == SB_F64 ? 8 : 4;
    uint32_t * tind[SB_MAX_NMODES] = {0};
    void * tval = NULL;
    uint64_t * counts = calloc(nt, sizeof(uint64_t));
    for(idx_t m = 0; m < nmodes && rc == SB_OK; ++m) {
      rc = sb_malloc((void **) &tind[m], nnz * sizeof(uint32_t));
    }
    if(rc == SB_OK) { rc = sb_malloc(&tval, nnz * vb); }
    if(rc == SB_OK) {
      rc = sb_tile_partition((uint32_t) nmodes, nnz, (uint32_t * const *) dind, dval, val_type,
          tsize, tdim, nt, tind, tval, counts);
    }
    uint64_t off = 0;
    for(idx_t t = 0; t < nt && rc == SB_OK; ++t) {
      if(counts[t] == 0) {                       /* empty tile */
        d[t].nmodes = (uint32_t) nmodes;
        d[t].val_type = val_type;
        for(idx_t m = 0; m < nmodes; ++m) { d[t].dims[m] = d64[m]; d[t].dim_perm[m] = p32[m]; }
        continue;
      }
      uint32_t * sub[SB_MAX_NMODES];
      for(idx_t m = 0; m < nmodes; ++m) { sub[m] = tind[m] + off; }
      rc = sb_csf_build((uint32_t) nmodes, counts[t], d64, sub, (char const *) tval + off * vb,
          val_type, p32, d + t);
      off += counts[t];
    }
    for(idx_t m = 0; m < nmodes; ++m) { sb_free(tind[m]); }
    sb_free(tval);
    free(counts);
  }
  if(rc) { return rc; }
  for(idx_t t = 0; t < nt; ++t) {
    for(idx_t l = 0; l < nmodes; ++l) { ct->pt[t].nfibs[l] = d[t].nfibs[l]; }
  }
  if(!mirror) { return SB_OK; }
  for(idx_t t = 0; t < nt && rc == SB_OK; ++t) {
    rc = p_mirror(ct->pt + t, d + t, nmodes, val_type, nt > 1);
  }
  return rc;
}

static void p_free_one(splatt_csf * ct)
{
  idx_t const nt = ct->ntiles ? ct->ntiles : 1;
  if(ct->pt) {
    for(idx_t t = 0; t < nt; ++t) {
      for(idx_t l = 0; l < ct->nmodes; ++l) { free(ct->pt[t].fptr[l]); free(ct->pt[t].fids[l]); }
      free(ct->pt[t].vals);
    }
    free(ct->pt);
    ct->pt = NULL;
  }
  if(ct->dev) {
    sb_dcsf * d = (sb_dcsf *) ct->dev;
    for(idx_t t = 0; t < nt; ++t) { sb_csf_release(d + t); }
    free(d);
    ct->dev = NULL;
  }
}

/* MTTKRP of one tree into `out` (zeroed first), summing its tiles */
int sb_tree_mttkrp(splatt_csf const * t, uint32_t out_level, uint32_t R,
    void * const * mats_by_level, uint32_t ld, void * out, uint32_t ld_out, int vt)
{
  sb_dcsf const * d = (sb_dcsf const *) t->dev;
  if(!d) { return SB_EINPUT; }
  int rc = SB_OK;
  for(idx_t k = 0; k < t->ntiles && rc == SB_OK; ++k) {
    if(k > 0 && d[k].nnz == 0) { continue; }
    if(d[k].val_type != vt) { return SB_EINPUT; }
    rc = sb_mttkrp_csf_acc(d + k, out_level, R, mats_by_level, ld, out, ld_out, vt, k == 0);
  }
  return rc;
}

/* sum of squared values over the tree's tiles */
int sb_tree_frobsq(splatt_csf const * t, double * out)
{
  sb_dcsf const * d = (sb_dcsf const *) t->dev;
  *out = 0.;
  if(!d) { return SB_EINPUT; }
  for(idx_t k = 0; k < t->ntiles; ++k) {
    if(d[k].nnz == 0) { continue; }
    double x = 0.;
    int const rc = sb_frobsq(d[k].vals, d[k].val_type, d[k].nnz, &x);
    if(rc) { return rc; }
    *out += x;
  }
  return SB_OK;
}

/* SPLATT_OPTION_TILE: untiled (NULL) or dense tiles (the options array) */
static int p_tiling(double const * opts, double const ** tile_opts)
{
  double const w = opts[SPLATT_OPTION_TILE];
  *tile_opts = NULL;
  if(w == SPLATT_NOTILE || w == SPLATT_VAL_OFF) { return SB_OK; }
  if(w == SPLATT_DENSETILE) { *tile_opts = opts; return SB_OK; }
  return SB_EINPUT;                              /* other schemes: not built */
}

/* common builder for csf_alloc / csf_convert; returns the tree array */
static splatt_error_type p_alloc(idx_t nmodes, idx_t nnz, idx_t const * dims,
    idx_t * const * inds, val_t const * vals, double const * opts, splatt_csf ** out,
    uint32_t ** keep_dind)
{
  *out = NULL;
  if(nmodes < 2 || nmodes > SPLATT_MAX_NMODES || nnz == 0 || nnz >= 0xffffffffull) {
    return SPLATT_ERROR_BADINPUT;
  }
  double const * tile_opts = NULL;
  if(p_tiling(opts, &tile_opts) != SB_OK) { return SPLATT_ERROR_BADINPUT; }
  int rc = sb_ensure_init();
  if(rc) { return sb_err(rc); }
  uint32_t * dind[SB_MAX_NMODES];
  void * dval = NULL;
  rc = sb_upload_coo(nmodes, nnz, dims, inds, vals, dind, &dval);
  if(rc) { return sb_err(rc); }

  int which = (int) opts[SPLATT_OPTION_CSF_ALLOC];
  idx_t const ncsf = which == SPLATT_CSF_ONEMODE ? 1 : (which == SPLATT_CSF_TWOMODE ? 2 : nmodes);
  splatt_csf * ret = calloc(ncsf, sizeof(*ret));
  idx_t perm[SPLATT_MAX_NMODES];
  if(which == SPLATT_CSF_ALLMODE) {
    for(idx_t m = 0; m < nmodes && rc == SB_OK; ++m) {
      sb_order_minusone(dims, nmodes, m, perm);
      rc = p_mk_csf(ret + m, nmodes, nnz, dims, dind, dval, perm, tile_opts);
    }
  } else {
    sb_order_small(dims, nmodes, perm);
    rc = p_mk_csf(ret, nmodes, nnz, dims, dind, dval, perm, tile_opts);
    if(rc == SB_OK && ncsf == 2) {
      sb_order_minusone(dims, nmodes, ret[0].dim_perm[nmodes-1], perm);
      /* TWOMODE's second tree is never tiled (src/csf.c:716-724) */
      rc = p_mk_csf(ret + 1, nmodes, nnz, dims, dind, dval, perm, NULL);
    }
  }
  sb_free(dval);
  for(idx_t m = 0; m < nmodes; ++m) {
    if(keep_dind) { keep_dind[m] = dind[m]; } else { sb_free(dind[m]); }
  }
  if(rc) {
    for(idx_t i = 0; i < ncsf; ++i) { p_free_one(ret + i); }
    free(ret);
    return sb_err(rc);
  }
  *out = ret;
  return SPLATT_SUCCESS;
}

/* trees from COO already on the device (uint32 indices, checked < dims) */
static splatt_error_type p_alloc_device(idx_t nmodes, idx_t nnz, idx_t const * dims,
    uint32_t * const * dind, void const * dval, int val_type, double const * opts,
    splatt_csf ** out, int mirror)
{
  *out = NULL;
  if(nmodes < 2 || nmodes > SPLATT_MAX_NMODES || nnz == 0 || nnz >= 0xffffffffull) {
    return SPLATT_ERROR_BADINPUT;
  }
  double const * tile_opts = NULL;
  if(p_tiling(opts, &tile_opts) != SB_OK) { return SPLATT_ERROR_BADINPUT; }
  int rc = sb_ensure_init();
  for(idx_t m = 0; m < nmodes && rc == SB_OK; ++m) {
    if(dims[m] >= 0xffffffffull) { return SPLATT_ERROR_BADINPUT; }
    rc = sb_check_u32(dind[m], nnz, dims[m]);
  }
  if(rc) { return sb_err(rc); }
  int which = (int) opts[SPLATT_OPTION_CSF_ALLOC];
  idx_t const ncsf = which == SPLATT_CSF_ONEMODE ? 1 : (which == SPLATT_CSF_TWOMODE ? 2 : nmodes);
  splatt_csf * ret = calloc(ncsf, sizeof(*ret));
  idx_t perm[SPLATT_MAX_NMODES];
  for(idx_t t = 0; t < ncsf && rc == SB_OK; ++t) {
    if(which == SPLATT_CSF_ALLMODE) {
      sb_order_minusone(dims, nmodes, t, perm);
    } else if(t == 0) {
      sb_order_small(dims, nmodes, perm);
    } else {
      sb_order_minusone(dims, nmodes, ret[0].dim_perm[nmodes-1], perm);
    }
    rc = p_mk_csf_typed(ret + t, nmodes, nnz, dims, dind, dval, perm, val_type, mirror,
        (which == SPLATT_CSF_TWOMODE && t == 1) ? NULL : tile_opts);
  }
  if(rc) {
    for(idx_t i = 0; i < ncsf; ++i) { p_free_one(ret + i); }
    free(ret);
    return sb_err(rc);
  }
  *out = ret;
  return SPLATT_SUCCESS;
}

splatt_error_type splatt_b200_csf_convert_device(uint32_t nmodes, uint64_t nnz,
    uint64_t const * dims, uint32_t * const * dinds, void const * dvals, int val_type,
    splatt_csf ** tensors, double const * const options, int host_mirror)
{
  if(!dims || !dinds || !dvals || !tensors || !options || nmodes > SPLATT_MAX_NMODES) {
    return SPLATT_ERROR_BADINPUT;
  }
  idx_t d[SPLATT_MAX_NMODES];
  for(uint32_t m = 0; m < nmodes; ++m) { d[m] = (idx_t) dims[m]; }
  return p_alloc_device(nmodes, nnz, d, dinds, dvals, val_type, options, tensors, host_mirror);
}

splatt_error_type splatt_csf_convert(splatt_idx_t const nmodes, splatt_idx_t const nnz,
    splatt_idx_t ** const inds, splatt_val_t * const vals, splatt_csf ** tensors,
    double const * const options)
{
  if(!inds || !vals || !tensors || !options || nmodes < 2 || nmodes > SPLATT_MAX_NMODES) {
    return SPLATT_ERROR_BADINPUT;
  }
  /* dimensions = 1 + the largest index of each mode */
  idx_t dims[SPLATT_MAX_NMODES];
  for(idx_t m = 0; m < nmodes; ++m) {
    idx_t mx = 0;
    for(idx_t n = 0; n < nnz; ++n) { if(inds[m][n] > mx) { mx = inds[m][n]; } }
    dims[m] = mx + 1;
  }
  return p_alloc(nmodes, nnz, dims, inds, vals, options, tensors, NULL);
}

splatt_csf * splatt_csf_alloc(splatt_coord * const tt, double const * const opts)
{
  splatt_csf * ret = NULL;
  if(p_alloc(tt->nmodes, tt->nnz, tt->dims, tt->ind, tt->vals, opts, &ret, NULL)
      != SPLATT_SUCCESS) {
    return NULL;
  }
  /* SPLATT sorts the caller's tensor in place (src/csf.c:387, and buckets
   * it by tile, src/tile.c:296-318); leave it in the order of the last tree
   * built, as SPLATT does */
  splatt_csf const * last = ret + sb_csf_count(ret, opts) - 1;
  sb_dcsf const * d = (sb_dcsf const *) last->dev;
  idx_t const N = tt->nmodes;
  idx_t base = 0;
  for(idx_t k = 0; k < last->ntiles; ++k) {
    csf_sparsity const * pt = last->pt + k;
    idx_t const tnnz = pt->nfibs[N-1];
    if(tnnz == 0) { continue; }
    for(idx_t n = 0; n < tnnz; ++n) {
      tt->ind[last->dim_perm[N-1]][base + n] = pt->fids[N-1][n];
      tt->vals[base + n] = pt->vals[n];
    }
    /* root ids: in the mirror when tiled, else on the device only (the
     * host mirror keeps SPLATT's NULL) */
    idx_t * root = pt->fids[0];
    idx_t * own = NULL;
    if(!root) {
      own = root = malloc(pt->nfibs[0] * sizeof(idx_t));
      if(p_d2h_idx(root, d[k].fids[0], pt->nfibs[0]) != SB_OK) {
        free(own);
        splatt_csf_free(ret, opts);
        return NULL;
      }
    }
    /* expand the upper levels back to per-nonzero coordinates */
    for(idx_t l = 0; l + 1 < N; ++l) {
      idx_t const mode = last->dim_perm[l];
      for(idx_t q0 = 0; q0 < pt->nfibs[l]; ++q0) {
        idx_t b = q0, e = q0 + 1;
        for(idx_t q = l; q + 1 < N; ++q) {
          b = pt->fptr[q][b];
          e = pt->fptr[q][e];
        }
        idx_t const id = (l == 0) ? root[q0] : pt->fids[l][q0];
        for(idx_t n = b; n < e; ++n) { tt->ind[mode][base + n] = id; }
      }
    }
    free(own);
    base += tnnz;
  }
  return ret;
}

void splatt_csf_free(splatt_csf * const csf, double const * const opts)
{
  if(!csf) { return; }
  idx_t const n = sb_csf_count(csf, opts);
  for(idx_t i = 0; i < n; ++i) { p_free_one(csf + i); }
  free(csf);
}

void splatt_free_csf(splatt_csf * tensors, double const * const options)
{
  splatt_csf_free(tensors, options);
}

splatt_error_type splatt_csf_load(char const * const fname, splatt_idx_t * nmodes,
    splatt_csf ** tensors, double const * const options)
{
  /* the file onto the device (parsed or converted there), empty slices
   * dropped there (tt_remove_empty), the CSF built from the device COO */
  if(!fname || !nmodes || !tensors || !options) { return SPLATT_ERROR_BADINPUT; }
  idx_t N = 0, nnz = 0, dims[SPLATT_MAX_NMODES];
  uint32_t * dind[SPLATT_MAX_NMODES] = {0};
  void * dval = NULL;
  int rc = sb_read_tensor_device(fname, &N, &nnz, dims, dind, &dval);
  uint64_t removed = 0, d64[SPLATT_MAX_NMODES];
  for(idx_t m = 0; m < N; ++m) { d64[m] = dims[m]; }
  if(rc == SB_OK) { rc = sb_remove_empty_device((uint32_t) N, nnz, d64, dind, NULL, &removed); }
  for(idx_t m = 0; m < N; ++m) { dims[m] = d64[m]; }
  splatt_error_type e = rc == SB_OK ? SPLATT_SUCCESS : sb_err(rc);
  if(e == SPLATT_SUCCESS) {
    e = p_alloc_device(N, nnz, dims, dind, dval, SB_VT, options, tensors, 1);
  }
  for(idx_t m = 0; m < N; ++m) { sb_free(dind[m]); }
  sb_free(dval);
  *nmodes = N;
  return e;
}

splatt_val_t splatt_csf_frobsq(splatt_csf const * const tensor)
{
  double s = 0.;
  if(tensor->dev) { sb_tree_frobsq(tensor, &s); }
  return (val_t) s;
}

splatt_error_type splatt_b200_csf_set_precision(splatt_csf * tensors,
    double const * const options, int val_type)
{
  idx_t const n = sb_csf_count(tensors, options);
  for(idx_t i = 0; i < n; ++i) {
    for(idx_t k = 0; k < tensors[i].ntiles; ++k) {
      sb_dcsf * d = (sb_dcsf *) tensors[i].dev + k;
      if(!tensors[i].dev || d->val_type == val_type) { continue; }
      if(d->nnz == 0) { d->val_type = val_type; continue; }
      void * nv = NULL;
      int rc = sb_malloc(&nv, d->nnz * (val_type == SB_F64 ? 8 : 4));
      if(rc == SB_OK) { rc = sb_convert_vals(d->vals, d->val_type, nv, val_type, d->nnz); }
      if(rc) { sb_free(nv); return sb_err(rc); }
      sb_free(d->vals);
      d->vals = nv;
      d->val_type = val_type;
    }
  }
  return SPLATT_SUCCESS;
}
