/*
 * stream.c -- streaming CPD: the per-slice handle and splatt_cpd_stream.
 *
 * Host mirror of StreamCPD::compute (src/cpd/stream/StreamCPD.cc:311-571)
 * and ParserSimple (src/cpd/stream/ParserSimple.cc:13-149):
 *  - slice dims: dims[m] = max(1 + largest index in the slice, previous);
 *  - grow_mats: rows that appear for the first time get glibc-rand values
 *    (fill_rand, mode order), Aold / duals start at zero;
 *  - the per-slice update runs on the device (k_stream.cu), either PLAIN
 *    (one launch per phase, host reads the ADMM / outer convergence flags)
 *    or FUSED (one persistent cooperative launch per slice);
 *  - the StreamCPD option overrides: tolerance 5e-2, 25 inner iterations,
 *    inner tolerance 7e-2 (StreamCPD.cc:366-368); non-streamed modes use the
 *    max-column-norm ADMM (StreamCPD.cc:326-337); the streamed mode the
 *    Frobenius regularisation.
 */
#include "sb_host.h"
#include "../kernels/kstream.h"
#include "sb_stream.h"
#include <time.h>

static size_t g_alloc_count;   /* bytes of the stream being allocated */

static int p_alloc_zero(void ** p, size_t bytes)
{
  g_alloc_count += bytes;
  int rc = sb_malloc(p, bytes);
  if(rc == SB_OK) { rc = sb_memset(*p, 0, bytes); }
  return rc;
}

splatt_b200_stream * splatt_b200_stream_alloc(splatt_idx_t nmodes, splatt_idx_t stream_mode,
    splatt_idx_t const * max_dims, splatt_idx_t rank, double forget, double reg,
    splatt_idx_t max_iterations, splatt_b200_precision precision, splatt_b200_exec exec)
{
  if(nmodes < 2 || nmodes > SPLATT_MAX_NMODES || stream_mode >= nmodes || rank == 0 ||
      rank > 64 || !max_dims) {
    return NULL;
  }
  if(sb_ensure_init() != SB_OK) { return NULL; }
  splatt_b200_stream * s = calloc(1, sizeof(*s));
  s->N = nmodes;
  s->sm = stream_mode;
  s->R = rank;
  s->vt = precision == SPLATT_B200_FP32 ? SB_F32 : SB_F64;
  s->vb = s->vt == SB_F64 ? 8 : 4;
  s->exec = exec;
  StreamArgs * a = &s->a;
  g_alloc_count = 0;
  a->N = (int) nmodes;
  a->sm = (int) stream_mode;
  a->R = (uint32_t) rank;
  a->nns = 0;
  idx_t maxcap = 1;
  for(idx_t m = 0; m < nmodes; ++m) {
    if(m == stream_mode) { continue; }
    a->ns[a->nns++] = (int) m;
    s->cap[m] = max_dims[m] > 0 ? max_dims[m] : 1;
    if(s->cap[m] > maxcap) { maxcap = s->cap[m]; }
  }
  a->reg = reg;
  a->forget = forget;
  a->outer_tol = 5e-2;
  a->inner_tol = 7e-2;
  a->max_outer = (int) max_iterations;
  a->max_inner = 25;
  size_t const R = rank;
  int rc = SB_OK;
  for(int q = 0; q < a->nns && rc == SB_OK; ++q) {
    int const m = a->ns[q];
    rc = p_alloc_zero(&a->Anew[m], s->cap[m] * R * s->vb);
    if(rc == SB_OK) { rc = p_alloc_zero(&a->Aold[m], s->cap[m] * R * s->vb); }
    if(rc == SB_OK) { rc = p_alloc_zero(&a->D[m], s->cap[m] * R * s->vb); }
  }
  for(idx_t m = 0; m < nmodes && rc == SB_OK; ++m) {
    rc = p_alloc_zero((void **) &a->G[m], R * R * sizeof(double));
  }
  if(rc == SB_OK) { rc = p_alloc_zero(&a->M, maxcap * R * s->vb); }
  if(rc == SB_OK) { rc = p_alloc_zero(&a->aux, maxcap * R * s->vb); }
  if(rc == SB_OK) { rc = p_alloc_zero(&a->init, maxcap * R * s->vb); }
  if(rc == SB_OK) { rc = p_alloc_zero((void **) &a->old_gram, R * R * sizeof(double)); }
  int const nh = a->nns > 1 ? a->nns - 1 : 1;
  if(rc == SB_OK) { rc = p_alloc_zero((void **) &a->H, nh * R * R * sizeof(double)); }
  if(rc == SB_OK) { rc = p_alloc_zero((void **) &a->Ginv, R * R * sizeof(double)); }
  if(rc == SB_OK) { rc = p_alloc_zero((void **) &a->s, R * sizeof(double)); }
  if(rc == SB_OK) { rc = p_alloc_zero(&a->sT, R * s->vb); }
  if(rc == SB_OK) { rc = p_alloc_zero((void **) &a->Mt, R * sizeof(double)); }
  s->nblocks = sb_stream_blocks((uint32_t) R, s->vt);
  if(rc == SB_OK) { rc = p_alloc_zero((void **) &a->red, SB_RED_SIZE * sizeof(double)); }
  if(rc == SB_OK) { rc = p_alloc_zero((void **) &a->bar, 2 * sizeof(unsigned)); }
  if(rc == SB_OK) { rc = p_alloc_zero((void **) &a->status, 12 * sizeof(int)); }
  if(rc == SB_OK) { rc = p_alloc_zero((void **) &s->d_err, sizeof(double)); }
  s->time_cap = 0;
  s->bytes = g_alloc_count;
  if(rc == SB_OK) { rc = sb_sync(); }
  if(rc) {
    splatt_b200_stream_free(s);
    return NULL;
  }
  return s;
}

void splatt_b200_stream_free(splatt_b200_stream * s)
{
  if(!s) { return; }
  StreamArgs * a = &s->a;
  for(idx_t m = 0; m < SPLATT_MAX_NMODES; ++m) {
    sb_free(a->Anew[m]); sb_free(a->Aold[m]); sb_free(a->D[m]); sb_free(a->G[m]);
    sb_free(s->dind[m]);
    sb_host_free(s->h_ind[m]);
  }
  sb_free(a->M); sb_free(a->aux); sb_free(a->init); sb_free(a->old_gram); sb_free(a->H);
  sb_free(a->Ginv); sb_free(a->s); sb_free(a->sT); sb_free(a->Mt);
  sb_free(a->red); sb_free(a->bar); sb_free(a->status);
  sb_free(s->dval); sb_free(s->d_time); sb_free(s->d_err);
  sb_host_free(s->h_val);
  free(s->h_rand);
  sb_sync();
  free(s);
}

splatt_error_type splatt_b200_stream_status(splatt_b200_stream const * s)
{
  if(!s) { return SPLATT_ERROR_BADINPUT; }
  return s->err ? (splatt_error_type) s->err : SPLATT_SUCCESS;
}

_Static_assert(SPLATT_B200_PROX_MAXCOLNORM == SB_PROX_MAXCOLNORM &&
               SPLATT_B200_PROX_MAXCOLNORM_NONNEG == SB_PROX_MAXCOLNORM_NONNEG &&
               SPLATT_B200_PROX_LASSO == SB_PROX_LASSO &&
               SPLATT_B200_PROX_ROWSIMP == SB_PROX_ROWSIMP &&
               SPLATT_B200_PROX_NTF_LASSO == SB_PROX_NTF_LASSO &&
               SPLATT_B200_PROX_NTF_FROB == SB_PROX_NTF_FROB &&
               SPLATT_B200_PROX_COLSIMP == SB_PROX_COLSIMP,
               "prox kinds shared with the kernels");

splatt_error_type splatt_b200_stream_set_prox(splatt_b200_stream * s, splatt_idx_t mode,
    splatt_b200_prox kind, double multiplier, splatt_idx_t chunk_rows)
{
  if(!s || mode >= (idx_t) s->N || mode == (idx_t) s->sm ||
      (kind != SPLATT_B200_PROX_MAXCOLNORM && kind != SPLATT_B200_PROX_MAXCOLNORM_NONNEG &&
       kind != SPLATT_B200_PROX_LASSO && kind != SPLATT_B200_PROX_ROWSIMP &&
       kind != SPLATT_B200_PROX_NTF_LASSO && kind != SPLATT_B200_PROX_NTF_FROB &&
       kind != SPLATT_B200_PROX_COLSIMP) ||
      !(multiplier >= 0.) || chunk_rows >= (1u << 30)) {
    return SPLATT_ERROR_BADINPUT;
  }
  s->a.prox[mode] = (int) kind;
  s->a.prox_mult[mode] = (kind == SPLATT_B200_PROX_LASSO || kind == SPLATT_B200_PROX_NTF_LASSO ||
                          kind == SPLATT_B200_PROX_NTF_FROB) ? multiplier : 0.;
  s->a.chunk[mode] = (uint32_t) (chunk_rows ? chunk_rows : 50);
  return SPLATT_SUCCESS;
}

splatt_idx_t splatt_b200_stream_last_outer(splatt_b200_stream const * s)
{
  return s ? s->last_outer : 0;
}

splatt_idx_t splatt_b200_stream_last_inner(splatt_b200_stream const * s, splatt_idx_t mode)
{
  if(!s) { return 0; }
  for(int q = 0; q < s->a.nns; ++q) {
    if((idx_t) s->a.ns[q] == mode) { return s->inner_mode[q]; }
  }
  return 0;
}

splatt_error_type splatt_b200_stream_sync(splatt_b200_stream * s)
{
  if(!s) { return SPLATT_ERROR_BADINPUT; }
  if(s->exec != SPLATT_B200_FUSED) { return sb_err(sb_sync()); }
  int st[12];
  int rc = sb_d2h(st, s->a.status, sizeof(st));
  if(rc) { return sb_err(rc); }
  if(st[0]) { s->err = SPLATT_ERROR_DEVICE; return SPLATT_ERROR_DEVICE; }
  s->last_outer = (idx_t) st[2];
  s->inner_total = (idx_t) st[3];
  for(int q = 0; q < s->a.nns; ++q) { s->inner_mode[q] = (idx_t) st[4 + q]; }
  return SPLATT_SUCCESS;
}

splatt_idx_t splatt_b200_stream_rows(splatt_b200_stream const * s, splatt_idx_t mode)
{
  return (s && mode < s->N) ? (mode == s->sm ? s->t : s->a.rows[mode]) : 0;
}

/* grow device slice buffers */
static int p_slice_room(splatt_b200_stream * s, idx_t nnz)
{
  if(nnz <= s->slice_cap) { return SB_OK; }
  idx_t cap = s->slice_cap ? s->slice_cap : 1024;
  while(cap < nnz) { cap *= 2; }
  int rc = SB_OK;
  for(idx_t m = 0; m < s->N && rc == SB_OK; ++m) {
    sb_free(s->dind[m]);
    s->dind[m] = NULL;
    sb_host_free(s->h_ind[m]);
    s->h_ind[m] = NULL;
    if(rc == SB_OK) { rc = sb_host_alloc((void **) &s->h_ind[m], cap * sizeof(uint32_t)); }
    if(m != s->sm) { rc = sb_malloc((void **) &s->dind[m], cap * sizeof(uint32_t)); }
  }
  sb_free(s->dval);
  s->dval = NULL;
  sb_host_free(s->h_val);
  s->h_val = NULL;
  if(rc == SB_OK) { rc = sb_host_alloc(&s->h_val, cap * s->vb); }
  if(rc == SB_OK) { rc = sb_malloc(&s->dval, cap * s->vb); }
  if(rc == SB_OK) { s->slice_cap = cap; }
  return rc;
}

int sbs_time_room(splatt_b200_stream * s)
{
  if(s->t < s->time_cap) { return SB_OK; }
  idx_t cap = s->time_cap ? 2 * s->time_cap : 256;
  double * nd = NULL;
  int rc = sb_malloc((void **) &nd, cap * s->R * sizeof(double));
  if(rc == SB_OK && s->t > 0) { rc = sb_d2d(nd, s->d_time, s->t * s->R * sizeof(double)); }
  if(rc) { sb_free(nd); return rc; }
  sb_free(s->d_time);
  s->d_time = nd;
  s->time_cap = cap;
  return SB_OK;
}

/* grow_mats (StreamCPD.cc:192-220): new rows drawn with rand() in mode
 * order, uploaded; Aold / D rows beyond the old count are still zero */
int sbs_grow(splatt_b200_stream * s, idx_t const * sdims)
{
  StreamArgs * a = &s->a;
  idx_t const R = s->R;
  int rc = SB_OK;
  for(int q = 0; q < a->nns && rc == SB_OK; ++q) {
    int const m = a->ns[q];
    idx_t const old = a->rows[m];
    a->rows0[m] = (uint32_t) old;
    if(sdims[m] > s->cap[m]) { return SB_EINPUT; }
    if(sdims[m] > old) {
      idx_t const n = (sdims[m] - old) * R;
      if(n > s->h_rand_cap) {
        free(s->h_rand);
        s->h_rand = malloc(n * sizeof(val_t));
        s->h_rand_cap = s->h_rand ? n : 0;
        if(!s->h_rand) { rc = SB_ENOMEM; break; }
      }
      if(s->private_rng) {
        for(idx_t i = 0; i < n; ++i) {
          val_t x = (val_t) (3.0 * ((val_t) rand_r(&s->rng_state) / (val_t) RAND_MAX));
          if(rand_r(&s->rng_state) % 2 == 0) { x = -x; }
          s->h_rand[i] = x;
        }
      } else {
        sb_fill_rand(s->h_rand, n);
      }
      if(s->vt == SB_VT) {
        rc = sb_h2d((char *) a->Anew[m] + old * R * s->vb, s->h_rand, n * s->vb);
      } else if(s->vt == SB_F32) {
        float * tmp = malloc(n * sizeof(float));
        if(!tmp) { rc = SB_ENOMEM; break; }
        for(idx_t i = 0; i < n; ++i) { tmp[i] = (float) s->h_rand[i]; }
        rc = sb_h2d((char *) a->Anew[m] + old * R * s->vb, tmp, n * sizeof(float));
        free(tmp);
      } else {
        double * tmp = malloc(n * sizeof(double));
        if(!tmp) { rc = SB_ENOMEM; break; }
        for(idx_t i = 0; i < n; ++i) { tmp[i] = (double) s->h_rand[i]; }
        rc = sb_h2d((char *) a->Anew[m] + old * R * s->vb, tmp, n * sizeof(double));
        free(tmp);
      }
      a->rows[m] = (uint32_t) sdims[m];
    }
  }
  return rc;
}

/* the PLAIN executor: one launch per phase, host-side control flow (the
 * ADMM and outer convergence tests read their sums back every time) */
static int p_run_plain(splatt_b200_stream * s)
{
  StreamArgs * a = &s->a;
  int const vt = s->vt, nb = s->nblocks;
  int rc = SB_OK;
  int k = 0;
#define PH(ph, mq, fl, ex) do { rc = sb_stream_phase(a, vt, (ph), (mq), (fl), (ex), k, nb); \
    if(rc) { return rc; } } while(0)
  for(int q = 0; q < a->nns; ++q) { PH(PH_GRAM, q, 0, 0); }
  if(a->first_slice) {
    for(int q = 0; q < a->nns; ++q) { PH(PH_NORM_PARTIAL, q, 0, 0); }
    for(int q = 0; q < a->nns; ++q) { PH(PH_NORM_APPLY, q, 0, 0); }
  }
  double prev = 0.;
  int outer;
  s->inner_total = 0;
  for(int q = 0; q < a->nns; ++q) { s->inner_mode[q] = 0; }
  for(outer = 0; outer < a->max_outer; ++outer) {
    PH(PH_TIME_MTTKRP, 0, 0, a->rows[a->ns[0]]);
    PH(PH_TIME_SOLVE, 0, 0, 0);
    for(int q = 0; q < a->nns; ++q) {
      PH(PH_MODE_MTTKRP, q, outer, 0);
      if(a->prox[a->ns[q]] == SB_PROX_COLSIMP) {
        /* single-chunk ADMM with the column simplex: the threshold rounds
         * run until no column's set above its threshold shrinks (the host
         * reads the counts after each round) */
        PH(PH_ADMM_FIRST, q, 1, 0);
        int it = 0;
        while(1) {
          int r = 0;
          double cnt[2][64];
          for(; r < 64; ++r) {
            PH(PH_COLSIMP_ROUND, q, r, 0);
            rc = sb_d2h(cnt[r & 1], a->red + SB_RD_SIMP + (r % SB_SIMP_RING) * 128 + 64, a->R * sizeof(double));
            if(rc) { return rc; }
            if(r > 0) {
              int done = 1;
              for(uint32_t c = 0; c < a->R; ++c) { if(cnt[r & 1][c] < cnt[(r - 1) & 1][c]) { done = 0; } }
              if(done) { break; }
            }
          }
          if(r == 64) { r = 63; }
          PH(PH_COLSIMP_APPLY, q, r, 0);
          double nrm[4];
          rc = sb_d2h(nrm, a->red + SB_RD_NRM + (k & 3) * 4, sizeof(nrm));
          if(rc) { return rc; }
          ++k;
          ++it;
          int const conv = (nrm[2] <= a->inner_tol * nrm[1]) && (nrm[3] <= a->inner_tol * nrm[0]);
          if(conv || it >= (int) a->max_inner) { break; }
          PH(PH_ADMM_FIRST, q, 0, 0);
        }
        s->inner_total += (idx_t) it;
        s->inner_mode[q] += (idx_t) it;
        uint32_t const next = (q + 1 < a->nns) ? a->rows[a->ns[q + 1]] : 0u;
        PH(PH_MODE_FINISH, q, outer, next);
        continue;
      }
      if(SB_PROX_CHUNKED(a->prox[a->ns[q]])) {
        /* row-separable: every chunk iterates to its own test in one launch */
        PH(PH_ADMM_CHUNKED, q, 0, 0);
        double tot = 0.;
        rc = sb_d2h(&tot, a->red + SB_RD_CHUNK + q, sizeof(tot));
        if(rc) { return rc; }
        idx_t const cum = (idx_t) llrint(tot / (double) a->rows[a->ns[q]]);
        s->inner_total += cum - s->inner_mode[q];
        s->inner_mode[q] = cum;
        uint32_t const next = (q + 1 < a->nns) ? a->rows[a->ns[q + 1]] : 0u;
        PH(PH_MODE_FINISH, q, outer, next);
        continue;
      }
      PH(PH_ADMM_FIRST, q, 1, 0);
      int it;
      for(it = 0; it < a->max_inner; ++it) {
        PH(PH_ADMM_SECOND, q, 0, 0);
        double nrm[4];
        rc = sb_d2h(nrm, a->red + SB_RD_NRM + (k & 3) * 4, sizeof(nrm));
        if(rc) { return rc; }
        ++k;
        /* src/cpd/admm.c:300-301 */
        int const conv = (nrm[2] <= a->inner_tol * nrm[1]) && (nrm[3] <= a->inner_tol * nrm[0]);
        if(conv || it + 1 == a->max_inner) { ++it; break; }
        PH(PH_ADMM_FIRST, q, 0, 0);
      }
      s->inner_total += (idx_t) it;
      s->inner_mode[q] += (idx_t) it;
      uint32_t const next = (q + 1 < a->nns) ? a->rows[a->ns[q + 1]] : 0u;
      PH(PH_MODE_FINISH, q, outer, next);
    }
    double dacc[16];
    rc = sb_d2h(dacc, a->red + SB_RD_DACC + (outer & 1) * 16, sizeof(dacc));
    if(rc) { return rc; }
    double delta = 0.;
    for(int q = 0; q < a->nns; ++q) { delta += sqrt(dacc[2 * q]) / sqrt(dacc[2 * q + 1]); }
    if(outer > 0 && fabs(delta - prev) < a->outer_tol) { ++outer; break; }
    prev = delta;
  }
  if(outer > a->max_outer) { outer = a->max_outer; }
  PH(PH_EPILOGUE, 0, outer, 0);
#undef PH
  s->last_outer = (idx_t) outer;
  return SB_OK;
}

/* per-slice clearing of the accumulators the phases add into */
static int p_clear(splatt_b200_stream * s)
{
  StreamArgs * a = &s->a;
  size_t const R = s->R;
  int rc = sb_memset(a->red, 0, SB_RED_SIZE * sizeof(double));
  if(rc == SB_OK) { rc = sb_memset(a->Mt, 0, R * sizeof(double)); }
  int const nh = a->nns > 1 ? a->nns - 1 : 1;
  if(rc == SB_OK) { rc = sb_memset(a->H, 0, nh * R * R * sizeof(double)); }
  for(int q = 0; q < a->nns && rc == SB_OK; ++q) {
    rc = sb_memset(a->G[a->ns[q]], 0, R * R * sizeof(double));
  }
  return rc;
}

void sbs_set_slice(splatt_b200_stream * s, uint32_t nnz, uint32_t * const * dinds, void * dvals)
{
  StreamArgs * a = &s->a;
  a->nnz = nnz;
  a->vals = dvals;
  for(idx_t m = 0; m < s->N; ++m) { a->inds[m] = dinds[m]; }
  a->first_slice = (s->t == 0);
  a->time_out = s->d_time + s->t * s->R;
  s->xnorm_last = -1.;   /* the slice's norm is taken on the device when asked for */
}

void sbs_advance(splatt_b200_stream * s) { ++s->t; }

int sbs_read_status(splatt_b200_stream * s)
{
  int st[12];
  int rc = sb_d2h(st, s->a.status, sizeof(st));
  if(rc) { return rc; }
  if(st[0]) { s->err = SPLATT_ERROR_DEVICE; return SB_EDEVICE; }
  s->last_outer = (idx_t) st[2];
  s->inner_total = (idx_t) st[3];
  for(int q = 0; q < s->a.nns; ++q) { s->inner_mode[q] = (idx_t) st[4 + q]; }
  return SB_OK;
}

void splatt_b200_stream_seed(splatt_b200_stream * s, unsigned seed)
{
  if(!s) { return; }
  s->private_rng = 1;
  s->rng_state = seed;
}

size_t splatt_b200_stream_bytes(splatt_b200_stream const * s) { return s ? s->bytes : 0; }

/* common driver once the slice is on the device */
static int p_step(splatt_b200_stream * s, uint32_t nnz, idx_t const * sdims, int sync_status)
{
  StreamArgs * a = &s->a;
  int rc = sbs_grow(s, sdims);
  if(rc) { return rc; }
  rc = sbs_time_room(s);
  if(rc) { return rc; }
  a->nnz = nnz;
  a->vals = s->dval;
  for(idx_t m = 0; m < s->N; ++m) { a->inds[m] = s->dind[m]; }
  a->first_slice = (s->t == 0);
  a->time_out = s->d_time + s->t * s->R;
  if(s->exec == SPLATT_B200_PLAIN) {
    rc = p_clear(s);          /* the fused kernel clears its own accumulators */
    if(rc) { return rc; }
  }
  if(s->exec == SPLATT_B200_FUSED) {
    rc = sb_stream_fused(a, s->vt, s->nblocks);
    if(rc == SB_OK && sync_status) {
      int st[12];
      rc = sb_d2h(st, a->status, sizeof(st));
      if(rc == SB_OK && st[0]) { rc = SB_EDEVICE; }
      s->last_outer = (idx_t) st[2];
      s->inner_total = (idx_t) st[3];
      for(int q = 0; q < a->nns; ++q) { s->inner_mode[q] = (idx_t) st[4 + q]; }
    }
  } else {
    rc = p_run_plain(s);
  }
  if(rc == SB_OK) { ++s->t; }
  return rc;
}

splatt_idx_t splatt_b200_stream_push(splatt_b200_stream * s, splatt_idx_t nnz,
    splatt_idx_t ** inds, splatt_val_t const * vals, splatt_val_t * time_row)
{
  if(!s || !inds || !vals || nnz == 0 || nnz >= 0xffffffffull) {
    if(s) { s->err = SPLATT_ERROR_BADINPUT; }
    return 0;
  }
  int rc = p_slice_room(s, nnz);
  if(rc) { s->err = sb_err(rc); return 0; }
  /* ParserSimple::next_batch dims + narrowing into the staging buffers */
  idx_t sdims[SPLATT_MAX_NMODES];
  for(idx_t m = 0; m < s->N; ++m) {
    if(m == s->sm) { sdims[m] = 1; continue; }
    idx_t mx = 0;
    idx_t const * src = inds[m];
    uint32_t * dst = s->h_ind[m];
    for(idx_t n = 0; n < nnz; ++n) {
      idx_t const x = src[n];
      if(x > mx) { mx = x; }
      dst[n] = (uint32_t) x;
    }
    sdims[m] = (mx + 1 > s->prevdim[m]) ? mx + 1 : s->prevdim[m];
    if(sdims[m] > s->cap[m]) { s->err = SPLATT_ERROR_BADINPUT; return 0; }
  }
  double xn = 0.;
  if(s->vt == SB_F64) {
    double * hv = s->h_val;
    for(idx_t n = 0; n < nnz; ++n) { hv[n] = (double) vals[n]; xn += (double) vals[n] * vals[n]; }
  } else {
    float * hv = s->h_val;
    for(idx_t n = 0; n < nnz; ++n) { hv[n] = (float) vals[n]; xn += (double) vals[n] * vals[n]; }
  }
  for(idx_t m = 0; m < s->N && rc == SB_OK; ++m) {
    if(m != s->sm) { rc = sb_h2d(s->dind[m], s->h_ind[m], nnz * sizeof(uint32_t)); }
  }
  if(rc == SB_OK) { rc = sb_h2d(s->dval, s->h_val, nnz * s->vb); }
  if(rc) { s->err = sb_err(rc); return 0; }
  for(idx_t m = 0; m < s->N; ++m) { if(m != s->sm) { s->prevdim[m] = sdims[m]; } }
  s->xnorm_last = xn;
  rc = p_step(s, (uint32_t) nnz, sdims, 1);
  if(rc) { s->err = sb_err(rc); return 0; }
  if(time_row) {
    double tr[64];
    rc = sb_d2h(tr, s->d_time + (s->t - 1) * s->R, s->R * sizeof(double));
    if(rc) { s->err = sb_err(rc); return 0; }
    for(idx_t r = 0; r < s->R; ++r) { time_row[r] = (val_t) tr[r]; }
  }
  return s->last_outer;
}

splatt_error_type splatt_b200_stream_push_device(splatt_b200_stream * s, splatt_idx_t nnz,
    uint32_t * const * dinds, void const * dvals, splatt_idx_t const * slice_dims)
{
  if(!s || !dinds || !dvals || !slice_dims || nnz == 0 || nnz >= 0xffffffffull) {
    return SPLATT_ERROR_BADINPUT;
  }
  idx_t sdims[SPLATT_MAX_NMODES];
  for(idx_t m = 0; m < s->N; ++m) {
    if(m == s->sm) { sdims[m] = 1; continue; }
    sdims[m] = slice_dims[m] > s->prevdim[m] ? slice_dims[m] : s->prevdim[m];
    if(sdims[m] > s->cap[m]) { return SPLATT_ERROR_BADINPUT; }
    s->prevdim[m] = sdims[m];
  }
  StreamArgs * a = &s->a;
  /* point the slice at the caller's device arrays */
  uint32_t * keep[SPLATT_MAX_NMODES];
  void * keepv = s->dval;
  for(idx_t m = 0; m < s->N; ++m) { keep[m] = s->dind[m]; s->dind[m] = dinds[m]; }
  s->dval = (void *) dvals;
  s->xnorm_last = -1.;
  int rc = p_step(s, (uint32_t) nnz, sdims, 0);
  for(idx_t m = 0; m < s->N; ++m) { s->dind[m] = keep[m]; }
  s->dval = keepv;
  (void) a;
  return rc ? sb_err(rc) : SPLATT_SUCCESS;
}

splatt_error_type splatt_b200_stream_factors(splatt_b200_stream * s, splatt_val_t ** factors,
    splatt_idx_t * rows)
{
  if(!s) { return SPLATT_ERROR_BADINPUT; }
  StreamArgs * a = &s->a;
  int rc = sb_sync();
  for(idx_t m = 0; m < s->N && rc == SB_OK; ++m) {
    idx_t const n = (m == s->sm) ? s->t : a->rows[m];
    if(rows) { rows[m] = n; }
    if(!factors || !factors[m] || n == 0) { continue; }
    size_t const cnt = n * s->R;
    if(m == s->sm) {
      double * tmp = malloc(cnt * sizeof(double));
      rc = sb_d2h(tmp, s->d_time, cnt * sizeof(double));
      for(size_t i = 0; i < cnt; ++i) { factors[m][i] = (val_t) tmp[i]; }
      free(tmp);
    } else if(s->vt == SB_VT) {
      rc = sb_d2h(factors[m], a->Anew[m], cnt * s->vb);
    } else if(s->vt == SB_F32) {
      float * tmp = malloc(cnt * sizeof(float));
      rc = sb_d2h(tmp, a->Anew[m], cnt * sizeof(float));
      for(size_t i = 0; i < cnt; ++i) { factors[m][i] = (val_t) tmp[i]; }
      free(tmp);
    } else {
      double * tmp = malloc(cnt * sizeof(double));
      rc = sb_d2h(tmp, a->Anew[m], cnt * sizeof(double));
      for(size_t i = 0; i < cnt; ++i) { factors[m][i] = (val_t) tmp[i]; }
      free(tmp);
    }
  }
  if(rc == SB_OK) {
    int st[12];
    rc = sb_d2h(st, a->status, sizeof(st));
    if(rc == SB_OK && st[0]) { return SPLATT_ERROR_DEVICE; }
  }
  return sb_err(rc);
}

double splatt_b200_stream_local_errsq(splatt_b200_stream * s)
{
  if(!s || s->t == 0) { return -1.; }
  double xn = s->xnorm_last;
  if(xn < 0.) {
    if(sb_frobsq(s->a.vals, s->vt, s->a.nnz, &xn) != SB_OK) { return -1.; }
  }
  double e = -1.;
  if(sb_stream_local_err(&s->a, s->vt, s->nblocks, xn, s->d_err) != SB_OK) { return -1.; }
  if(sb_d2h(&e, s->d_err, sizeof(double)) != SB_OK) { return -1.; }
  return e;
}

double splatt_b200_stream_window_errsq(splatt_b200_stream * s, splatt_idx_t nnz,
    uint32_t * const * dinds, double const * dvals, splatt_idx_t k)
{
  if(!s || s->t == 0 || !dinds || !dvals || k == 0 || nnz == 0 || nnz >= 0xffffffffull) {
    return -1.;
  }
  StreamArgs * a = &s->a;
  idx_t const R = s->R, N = s->N, T = s->t;
  idx_t const nk = k < T ? k : T, start = T - nk;
  double xn = 0.;
  int rc = sb_frobsq(dvals, SB_F64, nnz, &xn);
  /* <X, Z>: the COO MTTKRP of the window into the streamed mode (rows =
   * slices so far), dotted with the window's time rows; the factors in
   * FP64 (converted copies for an FP32 stream) */
  void * mats[SPLATT_MAX_NMODES] = {0};
  void * conv[SPLATT_MAX_NMODES] = {0};
  double * M = NULL;
  for(idx_t m = 0; m < N && rc == SB_OK; ++m) {
    if(m == s->sm) { mats[m] = s->d_time; continue; }
    if(s->vt == SB_F64) { mats[m] = a->Anew[m]; continue; }
    rc = sb_malloc(&conv[m], (a->rows[m] ? a->rows[m] : 1) * R * sizeof(double));
    if(rc == SB_OK) { rc = sb_convert_vals(a->Anew[m], SB_F32, conv[m], SB_F64, a->rows[m] * R); }
    mats[m] = conv[m];
  }
  if(rc == SB_OK) { rc = sb_malloc((void **) &M, T * R * sizeof(double)); }
  if(rc == SB_OK) {
    rc = sb_mttkrp_coo((uint32_t) N, nnz, dinds, dvals, (uint32_t) s->sm, (uint32_t) R,
        mats, (uint32_t) R, M, T, SB_F64);
  }
  double * hm = malloc(nk * R * sizeof(double));
  double * ht = malloc(nk * R * sizeof(double));
  double * hg = malloc(N * R * R * sizeof(double));
  if(!hm || !ht || !hg) { rc = SB_ENOMEM; }
  if(rc == SB_OK) { rc = sb_d2h(hm, M + start * R, nk * R * sizeof(double)); }
  if(rc == SB_OK) { rc = sb_d2h(ht, s->d_time + start * R, nk * R * sizeof(double)); }
  /* ||Z||^2 = sum_ij prod_m G_m(i,j): the maintained Grams of the factors
   * (upper triangles), and the window's time rows' Gram */
  for(idx_t m = 0; m < N && rc == SB_OK; ++m) {
    if(m != s->sm) { rc = sb_d2h(hg + m * R * R, a->G[m], R * R * sizeof(double)); }
  }
  double e = -1.;
  if(rc == SB_OK) {
    double inner = 0., zn = 0.;
    for(idx_t x = 0; x < nk * R; ++x) { inner += ht[x] * hm[x]; }
    for(idx_t i = 0; i < R; ++i) {
      for(idx_t j = i; j < R; ++j) {
        double gt = 0.;
        for(idx_t x = 0; x < nk; ++x) { gt += ht[x * R + i] * ht[x * R + j]; }
        double g = gt;
        for(idx_t m = 0; m < N; ++m) { if(m != s->sm) { g *= hg[m * R * R + i * R + j]; } }
        zn += (i == j) ? g : 2. * g;
      }
    }
    zn = fabs(zn);
    double const r = sqrt(xn + zn - 2. * inner) / sqrt(xn);
    e = r * r;
  }
  free(hm); free(ht); free(hg);
  sb_free(M);
  for(idx_t m = 0; m < N; ++m) { sb_free(conv[m]); }
  return e;
}

/* ---- splatt_cpd_stream: file in, mode%d.mat out --------------------------- */

static double p_wall(void)
{
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double) ts.tv_sec + 1e-9 * (double) ts.tv_nsec;
}

/* StreamCPD::compute's periodic full report (StreamCPD.cc:24-26, 521) */
#define SB_CHECK_ERR_INTERVAL 100

splatt_error_type splatt_cpd_stream(char const * const filename, splatt_idx_t rank,
    splatt_idx_t const stream_mode, double const forget, splatt_cpd_opts * const cpd_options,
    splatt_global_opts const * const global_options)
{
  /* the streaming kernels hold a rank-row in registers: R <= 64 */
  if(rank == 0 || rank > 64 || !filename) { return SPLATT_ERROR_BADINPUT; }
  /* the mode count from the file's first line or header; the options are
   * checked against it before any device work */
  idx_t N = 0, nnz = 0, fdims[SPLATT_MAX_NMODES];
  if(sb_file_modes(filename, &N) != SB_OK || stream_mode >= N) { return SPLATT_ERROR_BADINPUT; }
  uint32_t * dind[SPLATT_MAX_NMODES] = {0};
  void * dval = NULL;
  /* constraints as StreamCPD::compute maps them (StreamCPD.cc:325-337) */
  double reg = 0.;
  splatt_b200_prox prox[SPLATT_MAX_NMODES] = {SPLATT_B200_PROX_MAXCOLNORM};
  double pmult[SPLATT_MAX_NMODES] = {0.};
  for(idx_t m = 0; m < N; ++m) {
    splatt_cpd_constraint const * c = cpd_options ? cpd_options->constraints[m] : NULL;
    char const * d = c ? c->description : "UNCONSTRAINED";
    int ok = 1;
    if(m == stream_mode) {
      if(strncmp(d, "FROBENIUS", 9) == 0 && c && c->data) { reg = (double) *(val_t *) c->data; }
      else { ok = strcmp(d, "UNCONSTRAINED") == 0; }
    } else if(strcmp(d, "UNCONSTRAINED") == 0 || strcmp(d, "MAX-COL-NORM") == 0) {
      prox[m] = SPLATT_B200_PROX_MAXCOLNORM;
    } else if(strcmp(d, "NON-NEGATIVE") == 0 || strcmp(d, "NONNEG-MAX-COL-NORM") == 0) {
      prox[m] = SPLATT_B200_PROX_MAXCOLNORM_NONNEG;
    } else if(strncmp(d, "L1-REG", 6) == 0 && c && c->data) {
      prox[m] = SPLATT_B200_PROX_LASSO;
      pmult[m] = (double) *(val_t *) c->data;
    } else if(strcmp(d, "ROW-SIMPLEX") == 0) {
      prox[m] = SPLATT_B200_PROX_ROWSIMP;
    } else if(strcmp(d, "COL-SIMPLEX") == 0) {
      prox[m] = SPLATT_B200_PROX_COLSIMP;
    } else if(strncmp(d, "NTF-L1-REG", 10) == 0 && c && c->data) {
      /* both NTF registrations carry this description (nonneg_lasso.c:86,
       * nonneg_frob.c:92); the registration's marker tells them apart */
      prox[m] = sb_con_is_ntf_frob(c) ? SPLATT_B200_PROX_NTF_FROB : SPLATT_B200_PROX_NTF_LASSO;
      pmult[m] = (double) *(val_t *) c->data;
    } else {
      ok = 0;
    }
    if(!ok) { return SPLATT_ERROR_BADINPUT; }
  }
  /* the file onto the device (parsed or converted there) */
  idx_t N2 = 0;
  int const rrc = sb_read_tensor_device(filename, &N2, &nnz, fdims, dind, &dval);
  if(rrc != SB_OK || N2 != N) {
    for(idx_t m = 0; m < SPLATT_MAX_NMODES; ++m) { sb_free(dind[m]); }
    sb_free(dval);
    return rrc != SB_OK ? sb_err(rrc) : SPLATT_ERROR_BADINPUT;
  }
  if(global_options) { srand((unsigned) global_options->random_seed); }
  idx_t const T = fdims[stream_mode];
  /* ParserSimple's preparation on the device: order by (time, then the
   * following modes), relabel by first appearance, slice bounds */
  uint32_t * sind[SPLATT_MAX_NMODES] = {0};
  uint32_t * dmap[SPLATT_MAX_NMODES] = {0};
  void * dval64 = NULL, * sval = NULL;
  uint64_t d64[SPLATT_MAX_NMODES], nlab[SPLATT_MAX_NMODES] = {0};
  uint64_t * offs = calloc(T + 1, sizeof(uint64_t));
  uint64_t * seen = calloc(N * (T ? T : 1), sizeof(uint64_t));
  idx_t * iperm[SPLATT_MAX_NMODES] = {0};
  int rc = nnz > 0 && nnz < 0xffffffffull ? SB_OK : SB_EINPUT;
  for(idx_t m = 0; m < N; ++m) { d64[m] = fdims[m]; }
  if(rc == SB_OK && SB_VT != SB_F64) {                /* the stream runs in FP64 */
    rc = sb_malloc(&dval64, nnz * sizeof(double));
    if(rc == SB_OK) { rc = sb_convert_vals(dval, SB_VT, dval64, SB_F64, nnz); }
  }
  for(idx_t m = 0; m < N && rc == SB_OK; ++m) {
    rc = sb_malloc((void **) &sind[m], nnz * sizeof(uint32_t));
    if(rc == SB_OK && m != stream_mode) {
      rc = sb_malloc((void **) &dmap[m], fdims[m] * sizeof(uint32_t));
    }
  }
  if(rc == SB_OK) { rc = sb_malloc(&sval, nnz * sizeof(double)); }
  if(rc == SB_OK) {
    rc = sb_stream_prepare((uint32_t) N, nnz, d64, dind, dval64 ? dval64 : dval, SB_F64,
        (uint32_t) stream_mode, sind, sval, dmap, nlab, offs, seen);
  }
  for(idx_t m = 0; m < N; ++m) { sb_free(dind[m]); }
  sb_free(dval);
  sb_free(dval64);
  /* every time slice must be non-empty (ParserSimple.cc:113) */
  for(idx_t t = 0; t < T && rc == SB_OK; ++t) {
    if(offs[t + 1] == offs[t]) { rc = SB_EINPUT; }
  }
  for(idx_t m = 0; m < N && rc == SB_OK; ++m) {
    if(m == stream_mode) { continue; }
    iperm[m] = malloc((nlab[m] ? nlab[m] : 1) * sizeof(idx_t));
    uint32_t * tmp = malloc((nlab[m] ? nlab[m] : 1) * sizeof(uint32_t));
    rc = nlab[m] ? sb_d2h(tmp, dmap[m], nlab[m] * sizeof(uint32_t)) : SB_OK;
    for(idx_t i = 0; i < nlab[m]; ++i) { iperm[m][i] = tmp[i]; }
    free(tmp);
  }
  idx_t maxits = cpd_options ? cpd_options->max_iterations : 200;
  splatt_b200_stream * s = NULL;
  splatt_error_type ret = rc == SB_OK ? SPLATT_SUCCESS : sb_err(rc);
  if(ret == SPLATT_SUCCESS) {
    s = splatt_b200_stream_alloc(N, stream_mode, fdims, rank, forget, reg, maxits,
        SPLATT_B200_FP64, SPLATT_B200_FUSED);
    ret = s ? SPLATT_SUCCESS : SPLATT_ERROR_NOMEMORY;
  }
  for(idx_t m = 0; m < N && ret == SPLATT_SUCCESS; ++m) {
    if(m != stream_mode) {
      ret = splatt_b200_stream_set_prox(s, m, prox[m], pmult[m],
          cpd_options ? cpd_options->chunk_sizes[m] : 0);
    }
  }
  /* the reference's header (stream.cc:19-37) */
  printf("Streaming------------------------------------------------------\n");
  printf("STREAM-FILE=%s\n", filename);
  printf("STREAM-MODE=%" SPLATT_PF_IDX " STREAM-FORGET=%f RANK=%" SPLATT_PF_IDX
      " MAXITS=%" SPLATT_PF_IDX " TOL=%0.1e SEED=%d THREADS=%d\n", stream_mode + 1, forget,
      rank, maxits, cpd_options ? (double) cpd_options->tolerance : 1e-5,
      global_options ? global_options->random_seed : 0,
      global_options ? global_options->num_threads : 1);
  /* one slice per time index, straight from the device arrays; after each,
   * the driver's report line (StreamCPD.cc:509-534): local-1 every batch,
   * global (all slices so far) and local-10 every SB_CHECK_ERR_INTERVAL
   * batches and at the last; its "cpd" figure (a fresh CPD of the whole
   * history, compute_cpd_errorsq) is not computed here and prints -1 */
  idx_t t = 0;
  double stream_secs = 0.;
  for(; t < T && ret == SPLATT_SUCCESS; ++t) {
    uint32_t * bptr[SPLATT_MAX_NMODES];
    idx_t sd[SPLATT_MAX_NMODES];
    for(idx_t m = 0; m < N; ++m) {
      bptr[m] = sind[m] + offs[t];
      sd[m] = (m == stream_mode) ? 1 : (idx_t) seen[m * T + t];
    }
    idx_t const bnnz = offs[t + 1] - offs[t];
    double const t0 = p_wall();
    ret = splatt_b200_stream_push_device(s, bnnz, bptr, (double const *) sval + offs[t], sd);
    if(ret == SPLATT_SUCCESS) { ret = splatt_b200_stream_sync(s); }
    double const bsecs = p_wall() - t0;
    stream_secs += bsecs;
    if(ret != SPLATT_SUCCESS) { break; }
    idx_t const it = t + 1;
    double const local1 = splatt_b200_stream_local_errsq(s);
    double global = -1., local10 = -1.;
    if(it % SB_CHECK_ERR_INTERVAL == 0 || it == T) {
      uint32_t * wptr[SPLATT_MAX_NMODES];
      idx_t const w0 = it > 10 ? it - 10 : 0;
      for(idx_t m = 0; m < N; ++m) { wptr[m] = sind[m] + offs[w0]; }
      global = splatt_b200_stream_window_errsq(s, offs[it], sind, (double const *) sval, it);
      local10 = splatt_b200_stream_window_errsq(s, offs[it] - offs[w0], wptr,
          (double const *) sval + offs[w0], 10);
    }
    printf("batch %5" SPLATT_PF_IDX ": %7" SPLATT_PF_IDX " nnz (%0.5fs) (%0.3e NNZ/s) "
        "cpd: %+0.5f global: %+0.5f local-1: %+0.5f local-10: %+0.5f\n", it, bnnz, bsecs,
        (double) bnnz / bsecs, -1., global, local1, local10);
  }
  if(ret == SPLATT_SUCCESS) {
    printf("stream-time: %0.3fs\n", stream_secs);
    /* the final model on the whole stream (StreamCPD.cc:553-556) */
    double const fin = splatt_b200_stream_window_errsq(s, offs[t], sind, (double const *) sval, t);
    printf("\nfinal-err: %0.5f\n", fin);
    fflush(stdout);
  }
  for(idx_t m = 0; m < N; ++m) { sb_free(sind[m]); sb_free(dmap[m]); }
  sb_free(sval);
  free(offs);
  free(seen);
  /* write mode%d.mat in original row order (stream.cc:65-77) */
  if(ret == SPLATT_SUCCESS) {
    val_t * facs[SPLATT_MAX_NMODES] = {0};
    idx_t rows[SPLATT_MAX_NMODES];
    for(idx_t m = 0; m < N; ++m) {
      facs[m] = calloc((m == stream_mode ? t : fdims[m]) * rank + 1, sizeof(val_t));
    }
    ret = splatt_b200_stream_factors(s, facs, rows);
    for(idx_t m = 0; m < N && ret == SPLATT_SUCCESS; ++m) {
      char fname[64];
      sprintf(fname, "mode%" SPLATT_PF_IDX ".mat", m + 1);
      FILE * f = fopen(fname, "w");
      if(!f) { ret = SPLATT_ERROR_BADINPUT; break; }
      idx_t const nr = (m == stream_mode) ? rows[m] : fdims[m];
      /* rows that never appeared stay zero, as perm_matrix leaves them */
      val_t * out = calloc(nr * rank + 1, sizeof(val_t));
      for(idx_t i = 0; i < rows[m] && i < nr; ++i) {
        idx_t const dst = (m == stream_mode) ? i : iperm[m][i];
        memcpy(out + dst * rank, facs[m] + i * rank, rank * sizeof(val_t));
      }
      for(idx_t i = 0; i < nr; ++i) {
        for(idx_t r = 0; r < rank; ++r) { fprintf(f, "%+0.8e ", (double) out[i * rank + r]); }
        fprintf(f, "\n");
      }
      fclose(f);
      free(out);
    }
    for(idx_t m = 0; m < N; ++m) { free(facs[m]); }
  }
  splatt_b200_stream_free(s);
  for(idx_t m = 0; m < N; ++m) { free(iperm[m]); }
  return ret;
}
