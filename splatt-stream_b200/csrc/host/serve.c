/*
 * serve.c -- batched slice updates of many streams and the serving loop.
 *
 * No counterpart in SPLATT, whose streaming driver handles one tensor
 * (src/cpd/stream/StreamCPD.cc).  Each stream keeps StreamCPD's semantics;
 * what is added is running many independent streams on one GPU:
 *
 *  batch:  slices of many streams, several per stream allowed (a stream's
 *          slices form a chain and run in the order added), updated by one
 *          cooperative launch of the scheduled executor (k_stream_sched):
 *          the grid is cut into groups of g blocks; each group repeatedly
 *          claims the chain with the most slices left that no other group
 *          holds and runs its next slice with the fused update.  A slow
 *          slice (many outer / ADMM iterations) then holds one group while
 *          the others keep working, instead of holding a whole lockstep
 *          batch.  The launch (one H2D of the pinned argument block + the
 *          kernel) is captured once in a CUDA graph and replayed; two
 *          argument blocks alternate so a batch can be staged while the
 *          previous one runs.
 *  server: streams are admitted while their resident state fits an HBM
 *          budget; slices are queued per stream with their arrival time;
 *          every poll completes the batch in flight (non-blocking event
 *          query), admits waiting streams, and launches the next batch with
 *          every slice that has arrived (oldest stream first, up to the
 *          batch capacity) -- slices that arrive while a batch runs join
 *          the next one.  Per-slice latency = completion seen by the poll -
 *          arrival.
 *
 * Group size: g = max(1, blocks / chains) x f; the autotuner (g_tune)
 * chooses f in {1, 2, 4} per (precision, nnz bucket, rank bucket) by timing
 * the candidates on live batches; what it learns is kept for the process.
 */
#include "sb_stream.h"
#include <time.h>

typedef struct {
  void * h;                  /* pinned argument block (kstream.h layout) */
  void * d;                  /* device copy */
  void * graph;              /* captured H2D + launch (NULL: direct launches) */
} arg_block;

struct splatt_b200_batch {
  int vt;
  idx_t cap;                 /* slices per batch */
  int nblocks;
  uint32_t Rmax;
  size_t hdr_bytes;
  size_t bytes;
  arg_block blk[2];
  int cur;                   /* argument block being staged */
  int graph_ok;              /* -1 unknown, 0 unsupported, 1 in use */
  /* staged slices, in the order added */
  idx_t count;
  StreamArgs * it_args;
  splatt_b200_stream ** it_stream;
  idx_t * it_t;
  /* distinct streams of the batch staged / in flight in each block */
  splatt_b200_stream ** members[2];
  idx_t nmembers[2];
  void * ev[2];
  int inflight[2];
  int group;                 /* blocks per group; 0: automatic */
  int group_factor;          /* automatic size multiplier (autotuned) */
  int last_group;
};

splatt_b200_batch * splatt_b200_batch_alloc(splatt_idx_t max_slices,
    splatt_b200_precision precision, splatt_idx_t max_rank)
{
  if(max_slices == 0 || max_slices > (1u << 20) || max_rank == 0 || max_rank > 64 ||
      sb_ensure_init() != SB_OK) {
    return NULL;
  }
  splatt_b200_batch * b = calloc(1, sizeof(*b));
  b->vt = precision == SPLATT_B200_FP32 ? SB_F32 : SB_F64;
  b->cap = max_slices;
  b->Rmax = (uint32_t) max_rank;
  b->nblocks = sb_stream_blocks(b->Rmax, b->vt);
  if(b->nblocks > SB_SCHED_MAXG) { b->nblocks = SB_SCHED_MAXG; }
  b->hdr_bytes = SB_SCHED_HDR_BYTES(max_slices);
  b->bytes = b->hdr_bytes + max_slices * sizeof(StreamArgs);
  b->graph_ok = -1;
  b->group_factor = 1;
  b->it_args = calloc(max_slices, sizeof(StreamArgs));
  b->it_stream = calloc(max_slices, sizeof(*b->it_stream));
  b->it_t = calloc(max_slices, sizeof(idx_t));
  int rc = SB_OK;
  for(int i = 0; i < 2 && rc == SB_OK; ++i) {
    b->members[i] = calloc(max_slices, sizeof(*b->members[i]));
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
    free(b->members[i]);
  }
  sb_sync();
  free(b->it_args);
  free(b->it_stream);
  free(b->it_t);
  free(b);
}

void splatt_b200_batch_set_group(splatt_b200_batch * b, int blocks_per_group)
{
  if(b) { b->group = blocks_per_group > 0 ? blocks_per_group : 0; }
}

int splatt_b200_batch_last_group(splatt_b200_batch const * b) { return b ? b->last_group : 0; }

void splatt_b200_batch_set_factor(splatt_b200_batch * b, int factor)
{
  if(b) { b->group_factor = factor > 0 ? factor : 1; }
}

splatt_error_type splatt_b200_batch_add(splatt_b200_batch * b, splatt_b200_stream * s,
    splatt_idx_t nnz, uint32_t * const * dinds, void const * dvals,
    splatt_idx_t const * slice_dims)
{
  if(!b || !s || !dinds || !dvals || !slice_dims || nnz == 0 || nnz >= 0xffffffffull) {
    return SPLATT_ERROR_BADINPUT;
  }
  if(b->count == b->cap || s->vt != b->vt || s->R > b->Rmax || s->exec != SPLATT_B200_FUSED) {
    return SPLATT_ERROR_BADINPUT;
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
  /* New rows of a later slice in the chain are written now; the earlier
   * slices only touch rows below their own row counts. */
  int rc = sbs_grow(s, sdims);
  if(rc == SB_OK) { rc = sbs_time_room(s); }
  if(rc) { return sb_err(rc); }
  for(idx_t m = 0; m < s->N; ++m) { if(m != s->sm) { s->prevdim[m] = sdims[m]; } }
  sbs_set_slice(s, (uint32_t) nnz, dinds, (void *) dvals);
  b->it_args[b->count] = s->a;
  b->it_stream[b->count] = s;
  b->it_t[b->count] = s->t;
  ++b->count;
  sbs_advance(s);
  return SPLATT_SUCCESS;
}

/* write the staged slices into the pinned block as chains; returns chains */
static idx_t p_layout(splatt_b200_batch * b, int slot)
{
  int * h = (int *) b->blk[slot].h;
  memset(h, 0, b->hdr_bytes);
  splatt_b200_stream ** mem = b->members[slot];
  idx_t C = 0;
  idx_t * chain_of = malloc(b->count * sizeof(idx_t));
  int * len = h + 8 + b->cap;
  for(idx_t i = 0; i < b->count; ++i) {
    idx_t c = 0;
    while(c < C && mem[c] != b->it_stream[i]) { ++c; }
    if(c == C) { mem[C++] = b->it_stream[i]; }
    chain_of[i] = c;
    ++len[c];
  }
  int * base = h + 8;
  int * pos = calloc(C, sizeof(int));
  int acc = 0;
  for(idx_t c = 0; c < C; ++c) { base[c] = acc; acc += len[c]; }
  StreamArgs * items = (StreamArgs *) ((char *) h + b->hdr_bytes);
  for(idx_t i = 0; i < b->count; ++i) {
    idx_t const c = chain_of[i];
    StreamArgs * a = items + base[c] + pos[c]++;
    *a = b->it_args[i];
    /* the time history may have moved since the slice was staged */
    a->time_out = b->it_stream[i]->d_time + b->it_t[i] * b->it_stream[i]->R;
  }
  /* work estimate per chain (claim order): its slices' rows x R + nnz / 8 */
  double * w = calloc(C, sizeof(double));
  for(idx_t i = 0; i < b->count; ++i) {
    StreamArgs const * a = &b->it_args[i];
    double rows = 0.;
    for(int q = 0; q < a->nns; ++q) { rows += (double) a->rows[a->ns[q]]; }
    w[chain_of[i]] += rows * (double) a->R + (double) a->nnz / 8.;
  }
  int * prio = h + 8 + 4 * b->cap;
  double wtot = 0., wmax = 0.;
  for(idx_t c = 0; c < C; ++c) {
    double const x = w[c] / 64.;
    prio[c] = x > 2147483647. ? 2147483647 : (int) x;
    wtot += w[c];
    if(w[c] > wmax) { wmax = w[c]; }
  }
  free(pos);
  free(chain_of);
  b->nmembers[slot] = C;
  /* group layout.  Fixed size, or as many streams as blocks: uniform
   * groups (all take the heaviest chain first).  More streams than blocks:
   * a few large groups sized for the heaviest slice (its work times the
   * blocks over the total work) take the heavy chains, single blocks the
   * light ones. */
  int const nb = b->nblocks;
  int * gstart = h + 8 + 5 * b->cap + 3 * SB_SCHED_MAXG;
  int ng = 0, heavy = 1, gmax = 1;
  if(b->group > 0 || (int) C <= nb) {
    int g = b->group;
    if(g <= 0) {
      g = nb / (int) C;
      if(g < 1) { g = 1; }
      g *= b->group_factor;
    }
    if(g > nb) { g = nb; }
    ng = nb / g;
    for(int i = 0; i <= ng; ++i) { gstart[i] = i * g; }
    heavy = g;
    gmax = g;
  } else {
    int gb = (int) ceil(wmax * (double) nb / (wtot > 0. ? wtot : 1.)) * b->group_factor;
    if(gb < 1) { gb = 1; }
    if(gb > nb / 4) { gb = nb / 4 > 0 ? nb / 4 : 1; }
    int nheavy = 0;
    for(idx_t c = 0; c < C; ++c) { if(w[c] > wtot / (double) nb) { ++nheavy; } }
    int nbig = gb > 1 ? (nheavy < (nb / 2) / gb ? nheavy : (nb / 2) / gb) : 0;
    int at = 0;
    for(int i = 0; i < nbig; ++i) { gstart[ng++] = at; at += gb; }
    while(at < nb) { gstart[ng++] = at; at += 1; }
    gstart[ng] = at;
    heavy = nbig > 0 ? gb : 1;
    gmax = nbig > 0 ? gb : 1;
  }
  free(w);
  b->last_group = gmax;
  h[0] = (int) C;
  h[1] = heavy;
  h[2] = ng;
  h[3] = (int) b->cap;
  return C;
}

splatt_error_type splatt_b200_batch_run(splatt_b200_batch * b)
{
  if(!b || b->count == 0) { return SPLATT_ERROR_BADINPUT; }
  arg_block * k = &b->blk[b->cur];
  p_layout(b, b->cur);
  int rc = SB_OK;
  if(b->graph_ok != 0 && k->graph == NULL) {
    rc = sb_graph_capture_sched(&k->graph, k->d, k->h, b->bytes, b->vt, b->nblocks, b->Rmax);
    b->graph_ok = (rc == SB_OK) ? 1 : 0;
    rc = SB_OK;
  }
  if(b->graph_ok == 1) {
    rc = sb_graph_launch(k->graph);
  } else {
    rc = sb_h2d_async(k->d, k->h, b->bytes);
    if(rc == SB_OK) { rc = sb_stream_sched((int *) k->d, b->vt, b->nblocks, b->Rmax); }
  }
  if(rc == SB_OK) { rc = sb_event_record(b->ev[b->cur], NULL); }
  b->count = 0;
  if(rc) { return sb_err(rc); }
  b->inflight[b->cur] = 1;
  return SPLATT_SUCCESS;
}

/* completion bookkeeping of the batch launched from `slot` */
static splatt_error_type p_finish(splatt_b200_batch * b, int slot)
{
  sb_event_sync(b->ev[slot]);
  b->inflight[slot] = 0;
  splatt_error_type ret = SPLATT_SUCCESS;
  int err = 0;
  if(sb_d2h(&err, (char *) b->blk[slot].d + 4 * sizeof(int), sizeof(int)) != SB_OK || err) {
    ret = SPLATT_ERROR_DEVICE;
  }
  for(idx_t i = 0; i < b->nmembers[slot]; ++i) {
    if(sbs_read_status(b->members[slot][i]) != SB_OK) { ret = SPLATT_ERROR_DEVICE; }
  }
  b->nmembers[slot] = 0;
  return ret;
}

splatt_error_type splatt_b200_batch_sync(splatt_b200_batch * b)
{
  if(!b) { return SPLATT_ERROR_BADINPUT; }
  if(sb_sync() != SB_OK) { return SPLATT_ERROR_DEVICE; }
  splatt_error_type ret = p_finish(b, b->cur);
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
  idx_t inflight;             /* slices of this stream in the batch in flight */
  idx_t completed;
  int closed;
} srv_stream;

struct splatt_b200_server {
  int vt;
  size_t vb;
  size_t budget, used;
  idx_t max_batch;
  splatt_b200_batch * batch;
  srv_stream * st;
  idx_t nst, capst;
  int busy;
  idx_t * order;
  idx_t * take;
  /* slices in flight: stream and arrival */
  idx_t * fl_stream;
  double * fl_arrival;
  idx_t nfl;
  /* device arena holding the in-flight slices' COO */
  void * arena;
  size_t arena_cap;
  double * lat;
  idx_t nlat, caplat;
  idx_t batches;
  double batch_nnz;
  int cand;                   /* candidate of the batch in flight, -1: tuned */
  double launch_t;
};

/* Group-size autotuner, shared by every server of the process (what it
 * learns depends on the GPU and the workload, not on the server): per
 * (precision, nnz bucket, rank bucket) each candidate factor is timed on
 * two live batches (seconds per slice), then the fastest is kept. */
static int const g_factors[3] = {1, 2, 4};
static struct {
  int f[2][8][4];
  int done[2][8][4];
  double t[2][8][4][3];
  int n[2][8][4][3];
  int cand[2][8][4];
} g_tune;

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
  if(max_batch == 0) { return NULL; }
  splatt_b200_server * v = calloc(1, sizeof(*v));
  v->vt = precision == SPLATT_B200_FP32 ? SB_F32 : SB_F64;
  v->vb = v->vt == SB_F64 ? 8 : 4;
  v->budget = hbm_budget_bytes;
  v->max_batch = max_batch;
  v->batch = splatt_b200_batch_alloc(max_batch, precision, max_rank);
  if(!v->batch) { free(v); return NULL; }
  v->fl_stream = malloc(max_batch * sizeof(idx_t));
  v->fl_arrival = malloc(max_batch * sizeof(double));
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
  sb_free(v->arena);
  sb_sync();
  free(v->st);
  free(v->order);
  free(v->take);
  free(v->fl_stream);
  free(v->fl_arrival);
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
    v->take = realloc(v->take, v->capst * sizeof(idx_t));
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
  x->need = p_need(nmodes, stream_mode, max_dims, rank, v->vb);
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
  if(!v || id < 0 || (idx_t) id >= v->nst || nnz == 0 || nnz >= 0xffffffffull || !inds || !vals) {
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
    if(m == x->sm) { it->dims[m] = 1; continue; }   /* the time index is not uploaded */
    it->ind[m] = malloc(nnz * sizeof(uint32_t));
    idx_t mx = 0;
    for(idx_t n = 0; n < nnz; ++n) {
      idx_t const y = inds[m][n];
      if(y > mx) { mx = y; }
      it->ind[m][n] = (uint32_t) y;
    }
    it->dims[m] = mx + 1;
    if(it->dims[m] > x->max_dims[m]) {
      for(idx_t k = 0; k <= m; ++k) { free(it->ind[k]); }
      return SPLATT_ERROR_BADINPUT;
    }
  }
  it->vals = malloc(nnz * v->vb);
  for(idx_t n = 0; n < nnz; ++n) {
    if(v->vb == 8) { ((double *) it->vals)[n] = (double) vals[n]; }
    else { ((float *) it->vals)[n] = (float) vals[n]; }
  }
  ++x->qlen;
  return SPLATT_SUCCESS;
}

static size_t p_align(size_t x) { return (x + 255) & ~(size_t) 255; }

static size_t p_slice_bytes(splatt_b200_server const * v, srv_stream const * x, idx_t nnz)
{
  return (size_t) (x->N - 1) * p_align(nnz * sizeof(uint32_t)) + p_align(nnz * v->vb);
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

/* the batch in flight has finished: latencies, autotuner, bookkeeping */
static idx_t p_complete(splatt_b200_server * v, double now)
{
  splatt_b200_batch * b = v->batch;
  double const t = p_now() - v->launch_t;
  p_finish(b, b->cur);
  int const pv = v->vt == SB_F32, nb = p_bucket_nnz(v->batch_nnz), rb = p_bucket_rank(b->Rmax);
  int const c = v->cand;
  if(c >= 0 && !g_tune.done[pv][nb][rb] && g_tune.cand[pv][nb][rb] == c && v->nfl > 0) {
    g_tune.t[pv][nb][rb][c] += t / (double) v->nfl;
    if(++g_tune.n[pv][nb][rb][c] >= 2) {
      if(c == 2) {
        int best = 0;
        for(int k = 1; k < 3; ++k) {
          if(g_tune.t[pv][nb][rb][k] / g_tune.n[pv][nb][rb][k] <
             g_tune.t[pv][nb][rb][best] / g_tune.n[pv][nb][rb][best]) { best = k; }
        }
        g_tune.f[pv][nb][rb] = g_factors[best];
        g_tune.done[pv][nb][rb] = 1;
      }
      g_tune.cand[pv][nb][rb] = (c + 1) % 3;
    }
  }
  if(v->nlat + v->nfl > v->caplat) {
    while(v->nlat + v->nfl > v->caplat) { v->caplat = v->caplat ? 2 * v->caplat : 1024; }
    v->lat = realloc(v->lat, v->caplat * sizeof(double));
  }
  for(idx_t i = 0; i < v->nfl; ++i) {
    srv_stream * x = v->st + v->fl_stream[i];
    --x->inflight;
    ++x->completed;
    v->lat[v->nlat++] = now - v->fl_arrival[i];
  }
  idx_t const done = v->nfl;
  v->nfl = 0;
  b->cur ^= 1;
  v->busy = 0;
  return done;
}

splatt_idx_t splatt_b200_server_inflight(splatt_b200_server * v)
{
  if(!v || !v->busy) { return 0; }
  return sb_event_query_done(v->batch->ev[v->batch->cur]) ? 0 : (splatt_idx_t) v->nfl;
}

splatt_idx_t splatt_b200_server_poll(splatt_b200_server * v, double now)
{
  if(!v) { return 0; }
  splatt_b200_batch * b = v->batch;
  idx_t done = 0;
  /* 1. complete the batch in flight */
  if(v->busy) {
    if(sb_event_query_done(b->ev[b->cur]) == 0) { return 0; }
    done = p_complete(v, now);
  }
  /* 2. admission */
  p_admit(v);
  /* 3. next batch: every arrived slice, streams with the oldest head first */
  idx_t n = 0;
  for(idx_t i = 0; i < v->nst; ++i) {
    srv_stream * x = v->st + i;
    if(x->s && x->qlen > 0 && x->q[x->qhead].arrival <= now) { v->order[n++] = i; }
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
  /* take slices round-robin over the streams (one slice per stream per
   * round) so that a full batch spreads over as many streams as possible */
  idx_t * take = v->take;
  memset(take, 0, n * sizeof(idx_t));
  idx_t total = 0;
  size_t bytes = 0;
  for(int more = 1; more && total < v->max_batch;) {
    more = 0;
    for(idx_t k = 0; k < n && total < v->max_batch; ++k) {
      srv_stream * x = v->st + v->order[k];
      if(take[k] >= x->qlen) { continue; }
      slice_item * it = x->q + (x->qhead + take[k]) % x->qcap;
      if(it->arrival > now) { continue; }
      bytes += p_slice_bytes(v, x, it->nnz);
      ++take[k];
      ++total;
      more = 1;
    }
  }
  if(total == 0) { return done; }
  if(bytes > v->arena_cap) {
    sb_free(v->arena);
    v->arena = NULL;
    size_t cap = v->arena_cap ? v->arena_cap : ((size_t) 1 << 24);
    while(cap < bytes) { cap *= 2; }
    if(sb_malloc(&v->arena, cap) != SB_OK) { v->arena_cap = 0; return done; }
    v->arena_cap = cap;
  }
  char * cur = (char *) v->arena;
  double nnz_sum = 0.;
  for(idx_t k = 0; k < n; ++k) {
    srv_stream * x = v->st + v->order[k];
    for(idx_t r = 0; r < take[k]; ++r) {
      slice_item * it = x->q + x->qhead;
      uint32_t * dind[SPLATT_MAX_NMODES] = {NULL};
      int rc = SB_OK;
      for(idx_t m = 0; m < x->N && rc == SB_OK; ++m) {
        if(m == x->sm) { continue; }
        dind[m] = (uint32_t *) cur;
        rc = sb_h2d(cur, it->ind[m], it->nnz * sizeof(uint32_t));
        cur += p_align(it->nnz * sizeof(uint32_t));
      }
      void * dval = cur;
      if(rc == SB_OK) { rc = sb_h2d(cur, it->vals, it->nnz * v->vb); }
      cur += p_align(it->nnz * v->vb);
      if(rc != SB_OK) { break; }
      /* the time-mode index pointer is never read; give it a valid one */
      dind[x->sm] = dind[x->sm == 0 ? 1 : 0];
      if(splatt_b200_batch_add(b, x->s, it->nnz, dind, dval, it->dims) != SPLATT_SUCCESS) {
        break;
      }
      v->fl_stream[v->nfl] = v->order[k];
      v->fl_arrival[v->nfl] = it->arrival;
      ++v->nfl;
      ++x->inflight;
      nnz_sum += (double) it->nnz;
      p_pop(x);
    }
  }
  if(b->count == 0) { return done; }
  v->batch_nnz = nnz_sum / (double) b->count;
  int const pv = v->vt == SB_F32, nb = p_bucket_nnz(v->batch_nnz), rb = p_bucket_rank(b->Rmax);
  if(g_tune.done[pv][nb][rb] || b->group != 0) {
    v->cand = -1;
    b->group_factor = g_tune.done[pv][nb][rb] ? g_tune.f[pv][nb][rb] : 1;
  } else {
    v->cand = g_tune.cand[pv][nb][rb];
    b->group_factor = g_factors[v->cand];
  }
  v->launch_t = p_now();
  if(splatt_b200_batch_run(b) == SPLATT_SUCCESS) {
    v->busy = 1;
    ++v->batches;
  } else {
    /* nothing was launched: these slices are lost to their streams */
    for(idx_t i = 0; i < v->nfl; ++i) { --v->st[v->fl_stream[i]].inflight; }
    v->nfl = 0;
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
    int const was_busy = v->busy;
    splatt_b200_server_poll(v, t);
    if(!was_busy && !v->busy) { return SPLATT_ERROR_DEVICE; }   /* nothing could launch */
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
