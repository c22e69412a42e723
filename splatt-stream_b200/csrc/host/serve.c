/*
 * serve.c -- batched slice updates of many streams and the serving loop.
 *
 * No counterpart in SPLATT, whose streaming driver handles one tensor
 * (src/cpd/stream/StreamCPD.cc).  Each stream keeps StreamCPD's semantics;
 * what is added is running many independent streams on one GPU:
 *
 *  batch:  one slice from each of up to `max` streams, updated by a single
 *          cooperative launch (k_stream_batched): the grid is split into
 *          block groups sized by each stream's work, every group runs the
 *          fused slice update with its own group barrier.  The launch (one
 *          H2D of the pinned argument block + the kernel) is captured once
 *          in a CUDA graph and replayed; two argument blocks alternate so a
 *          batch can be staged while the previous one runs.
 *  server: streams are admitted while their resident state fits an HBM
 *          budget; slices are queued per stream with their arrival time;
 *          every poll completes the batch in flight (non-blocking event
 *          query), admits waiting streams, and launches the next batch from
 *          the streams that have a slice waiting (oldest first) -- slices
 *          that arrive while a batch runs join the next one.  Per-slice
 *          latency = completion seen by the poll - arrival.
 *
 * Block groups: a stream gets max(1, share of the grid proportional to its
 * work estimate rows*R + nnz/8) blocks; the autotuner (tune_*) chooses the
 * exponent of that weight per (nnz bucket, rank bucket) by timing the
 * candidates on live batches.
 */
#include "sb_stream.h"
#include <time.h>

#define SB_ARGS_ALIGN 256

typedef struct {
  void * h;                  /* pinned: int grp[max+2] | pad | StreamArgs[max] */
  void * d;                  /* device copy */
  void * graph;              /* captured H2D + launch (NULL: direct launches) */
} arg_block;

struct splatt_b200_batch {
  int vt;
  idx_t max;
  int nblocks;
  uint32_t Rmax;
  size_t grp_bytes;
  size_t bytes;
  arg_block blk[2];
  int cur;                   /* argument block being staged */
  int graph_ok;              /* -1 unknown, 0 unsupported, 1 in use */
  splatt_b200_stream ** members;
  idx_t count;
  void * ev[2];
  int inflight[2];
  double weight_exp;         /* group sizing weight exponent (autotuned) */
};

static size_t p_round(size_t x) { return (x + SB_ARGS_ALIGN - 1) / SB_ARGS_ALIGN * SB_ARGS_ALIGN; }

splatt_b200_batch * splatt_b200_batch_alloc(splatt_idx_t max_streams,
    splatt_b200_precision precision, splatt_idx_t max_rank)
{
  if(max_streams == 0 || max_rank == 0 || max_rank > 64 || sb_ensure_init() != SB_OK) {
    return NULL;
  }
  splatt_b200_batch * b = calloc(1, sizeof(*b));
  b->vt = precision == SPLATT_B200_FP32 ? SB_F32 : SB_F64;
  b->max = max_streams;
  b->Rmax = (uint32_t) max_rank;
  b->nblocks = sb_stream_blocks(b->Rmax, b->vt);
  b->grp_bytes = p_round((max_streams + 2) * sizeof(int));
  b->bytes = b->grp_bytes + max_streams * sizeof(StreamArgs);
  b->graph_ok = -1;
  b->weight_exp = 1.0;
  b->members = calloc(max_streams, sizeof(*b->members));
  int rc = SB_OK;
  for(int i = 0; i < 2 && rc == SB_OK; ++i) {
    rc = sb_host_alloc(&b->blk[i].h, b->bytes);
    if(rc == SB_OK) { rc = sb_malloc(&b->blk[i].d, b->bytes); }
    if(rc == SB_OK) { rc = sb_event_create(&b->ev[i]); }
  }
  if(rc == SB_OK) { rc = sb_sync(); }
  if(rc) { splatt_b200_batch_free(b); return NULL; }
  return b;
}

void splatt_b200_batch_free(splatt_b200_batch * b)
{
  if(!b) { return; }
  sb_sync();
  for(int i = 0; i < 2; ++i) {
    sb_graph_destroy(b->blk[i].graph);
    sb_host_free(b->blk[i].h);
    sb_free(b->blk[i].d);
    if(b->ev[i]) { sb_event_destroy(b->ev[i]); }
  }
  sb_sync();
  free(b->members);
  free(b);
}

void splatt_b200_batch_set_weight(splatt_b200_batch * b, double exponent)
{
  if(b) { b->weight_exp = exponent; }
}

splatt_error_type splatt_b200_batch_add(splatt_b200_batch * b, splatt_b200_stream * s,
    splatt_idx_t nnz, uint32_t * const * dinds, void const * dvals,
    splatt_idx_t const * slice_dims)
{
  if(!b || !s || !dinds || !dvals || !slice_dims || nnz == 0 || nnz >= 0xffffffffull) {
    return SPLATT_ERROR_BADINPUT;
  }
  if(b->count == b->max || s->vt != b->vt || s->R > b->Rmax) { return SPLATT_ERROR_BADINPUT; }
  for(idx_t i = 0; i < b->count; ++i) {
    if(b->members[i] == s) { return SPLATT_ERROR_BADINPUT; }   /* one slice per stream */
  }
  if(b->inflight[b->cur]) {
    /* the argument block we stage into is still read by a batch in flight */
    if(sb_event_sync(b->ev[b->cur]) != SB_OK) { return SPLATT_ERROR_DEVICE; }
    b->inflight[b->cur] = 0;
  }
  idx_t sdims[SPLATT_MAX_NMODES];
  for(idx_t m = 0; m < s->N; ++m) {
    if(m == s->sm) { sdims[m] = 1; continue; }
    sdims[m] = slice_dims[m] > s->prevdim[m] ? slice_dims[m] : s->prevdim[m];
    if(sdims[m] > s->cap[m]) { return SPLATT_ERROR_BADINPUT; }
  }
  int rc = sbs_grow(s, sdims);
  if(rc == SB_OK) { rc = sbs_time_room(s); }
  if(rc) { return sb_err(rc); }
  for(idx_t m = 0; m < s->N; ++m) { if(m != s->sm) { s->prevdim[m] = sdims[m]; } }
  sbs_set_slice(s, (uint32_t) nnz, dinds, (void *) dvals);
  StreamArgs * args = (StreamArgs *) ((char *) b->blk[b->cur].h + b->grp_bytes);
  args[b->count] = s->a;
  b->members[b->count++] = s;
  return SPLATT_SUCCESS;
}

/* block groups proportional to work^exp, at least one block each */
static void p_groups(splatt_b200_batch * b, int * grp)
{
  idx_t const S = b->count;
  int const nb = b->nblocks;
  grp[0] = (int) S;
  int * off = grp + 1;
  if((int) S > nb) {
    for(idx_t i = 0; i <= S; ++i) { off[i] = (int) i; }
    return;
  }
  double * w = malloc(S * sizeof(double));
  double tot = 0.;
  for(idx_t i = 0; i < S; ++i) {
    StreamArgs const * a = &b->members[i]->a;
    double rows = 0.;
    for(int q = 0; q < a->nns; ++q) { rows += (double) a->rows[a->ns[q]]; }
    double const work = rows * (double) a->R + (double) a->nnz / 8.;
    w[i] = pow(work > 1. ? work : 1., b->weight_exp);
    tot += w[i];
  }
  int const spare = nb - (int) S;
  int used = 0;
  int * cnt = malloc(S * sizeof(int));
  for(idx_t i = 0; i < S; ++i) {
    cnt[i] = 1 + (int) floor(spare * w[i] / tot);
    used += cnt[i];
  }
  /* leftover blocks to the heaviest streams */
  while(used < nb) {
    idx_t best = 0;
    double bw = -1.;
    for(idx_t i = 0; i < S; ++i) {
      double const per = w[i] / cnt[i];
      if(per > bw) { bw = per; best = i; }
    }
    ++cnt[best];
    ++used;
  }
  off[0] = 0;
  for(idx_t i = 0; i < S; ++i) { off[i + 1] = off[i] + cnt[i]; }
  free(cnt);
  free(w);
}

splatt_error_type splatt_b200_batch_run(splatt_b200_batch * b)
{
  if(!b || b->count == 0) { return SPLATT_ERROR_BADINPUT; }
  arg_block * k = &b->blk[b->cur];
  p_groups(b, (int *) k->h);
  StreamArgs const * dargs = (StreamArgs const *) ((char *) k->d + b->grp_bytes);
  int rc = SB_OK;
  if(b->graph_ok != 0 && k->graph == NULL) {
    rc = sb_graph_capture_batch(&k->graph, k->d, k->h, b->bytes, dargs, (int const *) k->d, b->vt,
        b->nblocks, b->Rmax);
    b->graph_ok = (rc == SB_OK) ? 1 : 0;
    rc = SB_OK;
  }
  if(b->graph_ok == 1) {
    rc = sb_graph_launch(k->graph);
  } else {
    rc = sb_h2d_async(k->d, k->h, b->bytes);
    if(rc == SB_OK) {
      rc = sb_stream_batched(dargs, (int const *) k->d, b->vt, b->nblocks, b->Rmax);
    }
  }
  if(rc == SB_OK) { rc = sb_event_record(b->ev[b->cur], NULL); }
  if(rc) { return sb_err(rc); }
  for(idx_t i = 0; i < b->count; ++i) { sbs_advance(b->members[i]); }
  b->inflight[b->cur] = 1;
  return SPLATT_SUCCESS;
}

/* members of the batch last launched, for completion bookkeeping */
static splatt_error_type p_finish(splatt_b200_batch * b, int slot)
{
  sb_event_sync(b->ev[slot]);
  b->inflight[slot] = 0;
  splatt_error_type ret = SPLATT_SUCCESS;
  for(idx_t i = 0; i < b->count; ++i) {
    if(sbs_read_status(b->members[i]) != SB_OK) { ret = SPLATT_ERROR_DEVICE; }
  }
  return ret;
}

splatt_error_type splatt_b200_batch_sync(splatt_b200_batch * b)
{
  if(!b) { return SPLATT_ERROR_BADINPUT; }
  if(sb_sync() != SB_OK) { return SPLATT_ERROR_DEVICE; }
  splatt_error_type ret = p_finish(b, b->cur);
  b->count = 0;
  b->cur ^= 1;
  return ret;
}

int splatt_b200_batch_graph_used(splatt_b200_batch const * b) { return b ? b->graph_ok : -1; }
int splatt_b200_batch_blocks(splatt_b200_batch const * b) { return b ? b->nblocks : 0; }

/* ========================================================================= */
/* serving loop                                                              */
/* ========================================================================= */

typedef struct {
  uint32_t * ind[SPLATT_MAX_NMODES];
  void * vals;
  idx_t nnz;
  idx_t dims[SPLATT_MAX_NMODES];
  double arrival;
} slice_item;

typedef struct {
  /* parameters */
  idx_t N, sm, R, maxits;
  idx_t max_dims[SPLATT_MAX_NMODES];
  double forget, reg;
  unsigned seed;
  /* state */
  splatt_b200_stream * s;     /* NULL until admitted */
  size_t need;
  slice_item * q;
  idx_t qhead, qlen, qcap;
  int inflight;
  double inflight_arrival;
  idx_t completed;
  int closed;
} srv_stream;

struct splatt_b200_server {
  int vt;
  size_t budget, used;
  idx_t max_batch;
  splatt_b200_batch * batch;
  srv_stream * st;
  idx_t nst, capst;
  int busy;
  idx_t * order;
  double * lat;
  idx_t nlat, caplat;
  idx_t batches;
  double batch_slices;
  /* autotuner: per (nnz bucket, rank bucket) best weight exponent */
  double tune_w[8][4];
  int tune_done[8][4];
  double tune_t[8][4][3];
  int tune_n[8][4][3];
  int tune_cand;
  double launch_t;
};

static double const g_weights[3] = {0.5, 1.0, 1.5};

/* device bytes a stream with these dims and rank will hold */
static size_t p_need(idx_t N, idx_t sm, idx_t const * dims, idx_t R, size_t vb)
{
  size_t rows = 0, maxrows = 1;
  for(idx_t m = 0; m < N; ++m) {
    if(m == sm) { continue; }
    rows += dims[m];
    if(dims[m] > maxrows) { maxrows = dims[m]; }
  }
  return (3 * rows + 3 * maxrows) * R * vb + (N + 8) * R * R * sizeof(double) + (1 << 16);
}

splatt_b200_server * splatt_b200_server_alloc(size_t hbm_budget_bytes,
    splatt_b200_precision precision, splatt_idx_t max_batch, splatt_idx_t max_rank)
{
  splatt_b200_server * v = calloc(1, sizeof(*v));
  v->vt = precision == SPLATT_B200_FP32 ? SB_F32 : SB_F64;
  v->budget = hbm_budget_bytes;
  v->max_batch = max_batch;
  v->batch = splatt_b200_batch_alloc(max_batch, precision, max_rank);
  if(!v->batch) { free(v); return NULL; }
  return v;
}

void splatt_b200_server_free(splatt_b200_server * v)
{
  if(!v) { return; }
  sb_sync();
  for(idx_t i = 0; i < v->nst; ++i) {
    srv_stream * x = v->st + i;
    for(idx_t k = 0; k < x->qlen; ++k) {
      slice_item * it = x->q + (x->qhead + k) % x->qcap;
      for(idx_t m = 0; m < x->N; ++m) { free(it->ind[m]); }
      free(it->vals);
    }
    free(x->q);
    splatt_b200_stream_free(x->s);
  }
  splatt_b200_batch_free(v->batch);
  free(v->st);
  free(v->order);
  free(v->lat);
  free(v);
}

int splatt_b200_server_open(splatt_b200_server * v, splatt_idx_t nmodes,
    splatt_idx_t stream_mode, splatt_idx_t const * max_dims, splatt_idx_t rank, double forget,
    double reg, splatt_idx_t max_iterations, unsigned seed)
{
  if(!v || nmodes < 2 || nmodes > SPLATT_MAX_NMODES || stream_mode >= nmodes || !max_dims) {
    return -1;
  }
  if(v->nst == v->capst) {
    v->capst = v->capst ? 2 * v->capst : 16;
    v->st = realloc(v->st, v->capst * sizeof(srv_stream));
    v->order = realloc(v->order, v->capst * sizeof(idx_t));
  }
  srv_stream * x = v->st + v->nst;
  memset(x, 0, sizeof(*x));
  x->N = nmodes;
  x->sm = stream_mode;
  x->R = rank;
  x->maxits = max_iterations;
  x->forget = forget;
  x->reg = reg;
  x->seed = seed;
  for(idx_t m = 0; m < nmodes; ++m) { x->max_dims[m] = max_dims[m]; }
  x->need = p_need(nmodes, stream_mode, max_dims, rank, v->vt == SB_F64 ? 8 : 4);
  return (int) v->nst++;
}

/* admit waiting streams while they fit the budget (in open order) */
static void p_admit(splatt_b200_server * v)
{
  for(idx_t i = 0; i < v->nst; ++i) {
    srv_stream * x = v->st + i;
    if(x->s || x->closed) { continue; }
    if(v->used + x->need > v->budget) { continue; }
    x->s = splatt_b200_stream_alloc(x->N, x->sm, x->max_dims, x->R, x->forget, x->reg, x->maxits,
        v->vt == SB_F32 ? SPLATT_B200_FP32 : SPLATT_B200_FP64, SPLATT_B200_FUSED);
    if(!x->s) { continue; }
    splatt_b200_stream_seed(x->s, x->seed);
    x->need = splatt_b200_stream_bytes(x->s) + 2 * 64 * 1024;
    v->used += x->need;
  }
}

splatt_error_type splatt_b200_server_close(splatt_b200_server * v, int id)
{
  if(!v || id < 0 || (idx_t) id >= v->nst) { return SPLATT_ERROR_BADINPUT; }
  srv_stream * x = v->st + id;
  if(x->inflight) { return SPLATT_ERROR_BADINPUT; }
  if(x->s) {
    splatt_b200_stream_free(x->s);
    x->s = NULL;
    v->used -= x->need;
  }
  x->closed = 1;
  return SPLATT_SUCCESS;
}

int splatt_b200_server_admitted(splatt_b200_server const * v, int id)
{
  return (v && id >= 0 && (idx_t) id < v->nst && v->st[id].s) ? 1 : 0;
}

splatt_error_type splatt_b200_server_submit(splatt_b200_server * v, int id, splatt_idx_t nnz,
    splatt_idx_t ** inds, splatt_val_t const * vals, double arrival)
{
  if(!v || id < 0 || (idx_t) id >= v->nst || nnz == 0 || !inds || !vals) {
    return SPLATT_ERROR_BADINPUT;
  }
  srv_stream * x = v->st + id;
  if(x->closed) { return SPLATT_ERROR_BADINPUT; }
  if(x->qlen == x->qcap) {
    idx_t const nc = x->qcap ? 2 * x->qcap : 8;
    slice_item * nq = malloc(nc * sizeof(slice_item));
    for(idx_t k = 0; k < x->qlen; ++k) { nq[k] = x->q[(x->qhead + k) % x->qcap]; }
    free(x->q);
    x->q = nq;
    x->qcap = nc;
    x->qhead = 0;
  }
  slice_item * it = x->q + (x->qhead + x->qlen) % x->qcap;
  memset(it, 0, sizeof(*it));
  it->nnz = nnz;
  it->arrival = arrival;
  for(idx_t m = 0; m < x->N; ++m) {
    it->ind[m] = malloc(nnz * sizeof(uint32_t));
    idx_t mx = 0;
    for(idx_t n = 0; n < nnz; ++n) {
      idx_t const y = inds[m][n];
      if(y > mx) { mx = y; }
      it->ind[m][n] = (uint32_t) y;
    }
    it->dims[m] = (m == x->sm) ? 1 : mx + 1;
    if(m != x->sm && it->dims[m] > x->max_dims[m]) {
      for(idx_t k = 0; k <= m; ++k) { free(it->ind[k]); }
      return SPLATT_ERROR_BADINPUT;
    }
  }
  size_t const vb = v->vt == SB_F64 ? 8 : 4;
  it->vals = malloc(nnz * vb);
  for(idx_t n = 0; n < nnz; ++n) {
    if(vb == 8) { ((double *) it->vals)[n] = (double) vals[n]; }
    else { ((float *) it->vals)[n] = (float) vals[n]; }
  }
  ++x->qlen;
  return SPLATT_SUCCESS;
}

/* upload the head slice of stream x into its device slice buffers */
static int p_upload_head(splatt_b200_server * v, srv_stream * x)
{
  splatt_b200_stream * s = x->s;
  slice_item * it = x->q + x->qhead;
  size_t const vb = v->vt == SB_F64 ? 8 : 4;
  int rc = SB_OK;
  if(it->nnz > s->dslice_cap) {
    idx_t cap = s->dslice_cap ? s->dslice_cap : 1024;
    while(cap < it->nnz) { cap *= 2; }
    for(idx_t m = 0; m < s->N; ++m) { sb_free(s->dslice[m]); s->dslice[m] = NULL; }
    sb_free(s->dslice_val);
    s->dslice_val = NULL;
    for(idx_t m = 0; m < s->N && rc == SB_OK; ++m) {
      if(m != s->sm) { rc = sb_malloc((void **) &s->dslice[m], cap * sizeof(uint32_t)); }
    }
    if(rc == SB_OK) { rc = sb_malloc(&s->dslice_val, cap * vb); }
    if(rc) { return rc; }
    s->dslice_cap = cap;
  }
  for(idx_t m = 0; m < s->N && rc == SB_OK; ++m) {
    if(m != s->sm) { rc = sb_h2d(s->dslice[m], it->ind[m], it->nnz * sizeof(uint32_t)); }
  }
  if(rc == SB_OK) { rc = sb_h2d(s->dslice_val, it->vals, it->nnz * vb); }
  return rc;
}

static void p_pop(srv_stream * x)
{
  slice_item * it = x->q + x->qhead;
  for(idx_t m = 0; m < x->N; ++m) { free(it->ind[m]); }
  free(it->vals);
  x->qhead = (x->qhead + 1) % x->qcap;
  --x->qlen;
}

static double p_now(void)
{
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static int p_bucket_nnz(double nnz)
{
  int b = 0;
  while(nnz >= 4096. && b < 7) { nnz /= 4.; ++b; }
  return b;
}

static int p_bucket_rank(idx_t R)
{
  return R <= 8 ? 0 : (R <= 16 ? 1 : (R <= 32 ? 2 : 3));
}

splatt_idx_t splatt_b200_server_poll(splatt_b200_server * v, double now)
{
  if(!v) { return 0; }
  splatt_b200_batch * b = v->batch;
  idx_t done = 0;
  /* 1. complete the batch in flight */
  if(v->busy) {
    int const q = sb_event_query_done(b->ev[b->cur]);
    if(q == 0) { return 0; }
    double const t = p_now() - v->launch_t;
    p_finish(b, b->cur);
    /* autotuner bookkeeping: time per slice of this batch */
    int const nb = p_bucket_nnz(v->batch_slices), rb = p_bucket_rank(b->Rmax);
    if(!v->tune_done[nb][rb]) {
      v->tune_t[nb][rb][v->tune_cand] += t / (double) b->count;
      if(++v->tune_n[nb][rb][v->tune_cand] >= 2) {
        if(v->tune_cand == 2) {
          int best = 0;
          for(int c = 1; c < 3; ++c) {
            if(v->tune_t[nb][rb][c] / v->tune_n[nb][rb][c] <
               v->tune_t[nb][rb][best] / v->tune_n[nb][rb][best]) { best = c; }
          }
          v->tune_w[nb][rb] = g_weights[best];
          v->tune_done[nb][rb] = 1;
        }
        v->tune_cand = (v->tune_cand + 1) % 3;
      }
    }
    for(idx_t i = 0; i < v->nst; ++i) {
      srv_stream * x = v->st + i;
      if(!x->inflight) { continue; }
      x->inflight = 0;
      ++x->completed;
      if(v->nlat == v->caplat) {
        v->caplat = v->caplat ? 2 * v->caplat : 1024;
        v->lat = realloc(v->lat, v->caplat * sizeof(double));
      }
      v->lat[v->nlat++] = now - x->inflight_arrival;
      ++done;
    }
    b->count = 0;
    b->cur ^= 1;
    v->busy = 0;
  }
  /* 2. admission */
  p_admit(v);
  /* 3. next batch: streams with a waiting slice, oldest arrival first */
  idx_t n = 0;
  for(idx_t i = 0; i < v->nst; ++i) {
    srv_stream * x = v->st + i;
    if(x->s && x->qlen > 0 && !x->inflight && x->q[x->qhead].arrival <= now) { v->order[n++] = i; }
  }
  if(n == 0) { return done; }
  for(idx_t a = 1; a < n; ++a) {          /* insertion sort by head arrival */
    idx_t const key = v->order[a];
    double const ka = v->st[key].q[v->st[key].qhead].arrival;
    idx_t j = a;
    while(j > 0 && v->st[v->order[j-1]].q[v->st[v->order[j-1]].qhead].arrival > ka) {
      v->order[j] = v->order[j-1];
      --j;
    }
    v->order[j] = key;
  }
  if(n > v->max_batch) { n = v->max_batch; }
  double nnz_sum = 0.;
  for(idx_t k = 0; k < n; ++k) {
    srv_stream * x = v->st + v->order[k];
    slice_item * it = x->q + x->qhead;
    if(p_upload_head(v, x) != SB_OK) { continue; }
    if(splatt_b200_batch_add(b, x->s, it->nnz, x->s->dslice, x->s->dslice_val, it->dims)
        != SPLATT_SUCCESS) {
      continue;
    }
    x->inflight = 1;
    x->inflight_arrival = it->arrival;
    nnz_sum += (double) it->nnz;
    p_pop(x);
  }
  if(b->count == 0) { return done; }
  v->batch_slices = nnz_sum / (double) b->count;
  int const nb = p_bucket_nnz(v->batch_slices), rb = p_bucket_rank(b->Rmax);
  b->weight_exp = v->tune_done[nb][rb] ? v->tune_w[nb][rb] : g_weights[v->tune_cand];
  v->launch_t = p_now();
  if(splatt_b200_batch_run(b) == SPLATT_SUCCESS) {
    v->busy = 1;
    ++v->batches;
  }
  return done;
}

splatt_error_type splatt_b200_server_drain(splatt_b200_server * v, double now)
{
  if(!v) { return SPLATT_ERROR_BADINPUT; }
  for(;;) {
    p_admit(v);
    int pending = v->busy;
    for(idx_t i = 0; i < v->nst && !pending; ++i) {
      if(v->st[i].s && v->st[i].qlen > 0) { pending = 1; }
    }
    if(!pending) { break; }
    if(v->busy) { sb_stream_sync(sb_get_stream()); }
    /* launch every queued slice regardless of its arrival time */
    double const t = (now > 0. ? now : p_now());
    for(idx_t i = 0; i < v->nst; ++i) {
      srv_stream * x = v->st + i;
      for(idx_t k = 0; k < x->qlen; ++k) {
        slice_item * it = x->q + (x->qhead + k) % x->qcap;
        if(it->arrival > t) { it->arrival = t; }
      }
    }
    splatt_b200_server_poll(v, t);
  }
  return SPLATT_SUCCESS;
}

splatt_error_type splatt_b200_server_stats(splatt_b200_server const * v, double * p50,
    double * p99, splatt_idx_t * completed, splatt_idx_t * batches)
{
  if(!v) { return SPLATT_ERROR_BADINPUT; }
  double * c = malloc((v->nlat ? v->nlat : 1) * sizeof(double));
  memcpy(c, v->lat, v->nlat * sizeof(double));
  for(idx_t a = 1; a < v->nlat; ++a) {
    double const key = c[a];
    idx_t j = a;
    while(j > 0 && c[j-1] > key) { c[j] = c[j-1]; --j; }
    c[j] = key;
  }
  if(p50) { *p50 = v->nlat ? c[(idx_t) (0.50 * (v->nlat - 1))] : 0.; }
  if(p99) { *p99 = v->nlat ? c[(idx_t) (0.99 * (v->nlat - 1))] : 0.; }
  if(completed) { *completed = v->nlat; }
  if(batches) { *batches = v->batches; }
  free(c);
  return SPLATT_SUCCESS;
}

void splatt_b200_server_reset_stats(splatt_b200_server * v)
{
  if(v) { v->nlat = 0; v->batches = 0; }
}

splatt_b200_stream * splatt_b200_server_stream(splatt_b200_server * v, int id)
{
  return (v && id >= 0 && (idx_t) id < v->nst) ? v->st[id].s : NULL;
}

size_t splatt_b200_server_used(splatt_b200_server const * v) { return v ? v->used : 0; }
