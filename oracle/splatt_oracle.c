/*
 * splatt_oracle.c -- CPU restatement of the SPLATT hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA path.  Never
 * linked into or called by the product library.  Single-threaded, written for
 * clarity rather than speed; every routine cites the reference function
 * (path:line within the SPLATT source tree) whose algorithm it restates.
 */
#include "splatt_oracle.h"
#include <stdlib.h>
#include <string.h>
#include <math.h>

typedef uint64_t u64;

/* ------------------------------------------------------------------------ */
/* factor initialisation: src/util.c:15-40 (rand_val / fill_rand)            */
/* value = 3 * rand()/RAND_MAX, negated when the next rand() is even.        */
/* ------------------------------------------------------------------------ */
static void orc_fill_rand(double * v, u64 n)
{
  for(u64 i = 0; i < n; ++i) {
    double x = 3.0 * ((double) rand() / (double) RAND_MAX);
    if(rand() % 2 == 0) { x = -x; }
    v[i] = x;
  }
}

/* ------------------------------------------------------------------------ */
/* mode orderings: src/csf.c:93-218, 608-651                                 */
/* SMALLFIRST = modes by ascending length (ties keep mode order);            */
/* MINUSONE   = `special` first, the rest by ascending length.               */
/* ------------------------------------------------------------------------ */
static void orc_order_small(u64 const * dims, u64 nmodes, u64 * perm)
{
  for(u64 m = 0; m < nmodes; ++m) { perm[m] = m; }
  for(u64 i = 1; i < nmodes; ++i) {          /* stable insertion sort */
    u64 x = perm[i];
    u64 j = i;
    while(j > 0 && dims[perm[j-1]] > dims[x]) { perm[j] = perm[j-1]; --j; }
    perm[j] = x;
  }
}

static void orc_order_minusone(u64 const * dims, u64 nmodes, u64 special,
    u64 * perm)
{
  u64 tmp[ORC_MAX_NMODES];
  orc_order_small(dims, nmodes, tmp);
  perm[0] = special;
  u64 k = 1;
  for(u64 m = 0; m < nmodes; ++m) {
    if(tmp[m] != special) { perm[k++] = tmp[m]; }
  }
}

/* ------------------------------------------------------------------------ */
/* lexicographic sort under a mode permutation: src/sort.c:761-956           */
/* (counting sort on the first mode + per-slice quicksort = a full           */
/* lexicographic order, unique for distinct coordinates).                    */
/* ------------------------------------------------------------------------ */
static u64 const * const * g_sort_inds;
static u64 const * g_sort_perm;
static u64 g_sort_nmodes;

static int orc_cmp(void const * a, void const * b)
{
  u64 const x = *(u64 const *) a;
  u64 const y = *(u64 const *) b;
  for(u64 l = 0; l < g_sort_nmodes; ++l) {
    u64 const * ind = g_sort_inds[g_sort_perm[l]];
    if(ind[x] != ind[y]) { return ind[x] < ind[y] ? -1 : 1; }
  }
  return x < y ? -1 : (x > y);
}

static u64 * orc_sorted_order(u64 nmodes, u64 nnz, u64 * const * inds,
    u64 const * perm)
{
  u64 * order = malloc(nnz * sizeof(u64));
  for(u64 n = 0; n < nnz; ++n) { order[n] = n; }
  g_sort_inds = (u64 const * const *) inds;
  g_sort_perm = perm;
  g_sort_nmodes = nmodes;
  qsort(order, nnz, sizeof(u64), orc_cmp);
  return order;
}

/* ------------------------------------------------------------------------ */
/* CSF construction: src/csf.c:230-416 (p_mk_outerptr, p_mk_fptr,           */
/* p_csf_alloc_untiled).  A node starts at level l wherever the coordinate  */
/* prefix (levels 0..l) changes; fptr[l] points into level l+1 (or into the  */
/* nonzeros at the last internal level).                                     */
/* ------------------------------------------------------------------------ */
static void orc_build_one(orc_csf * c, u64 nmodes, u64 nnz, u64 const * dims,
    u64 * const * inds, double const * vals, u64 const * perm)
{
  c->nmodes = nmodes;
  c->nnz = nnz;
  for(u64 m = 0; m < nmodes; ++m) {
    c->dims[m] = dims[m];
    c->dim_perm[m] = perm[m];
  }
  u64 * order = orc_sorted_order(nmodes, nnz, inds, perm);

  /* sorted coordinates by level */
  u64 * lv[ORC_MAX_NMODES];
  for(u64 l = 0; l < nmodes; ++l) {
    lv[l] = malloc(nnz * sizeof(u64));
    for(u64 n = 0; n < nnz; ++n) { lv[l][n] = inds[perm[l]][order[n]]; }
  }
  c->vals = malloc(nnz * sizeof(double));
  for(u64 n = 0; n < nnz; ++n) { c->vals[n] = vals[order[n]]; }

  /* first level at which position n differs from n-1 */
  u64 * first = malloc(nnz * sizeof(u64));
  for(u64 n = 0; n < nnz; ++n) {
    u64 l = 0;
    if(n > 0) {
      while(l < nmodes - 1 && lv[l][n] == lv[l][n-1]) { ++l; }
    }
    first[n] = l;
  }

  /* node numbering per level */
  for(u64 l = 0; l < nmodes; ++l) {
    u64 cnt = 0;
    for(u64 n = 0; n < nnz; ++n) { cnt += (l == nmodes - 1) || first[n] <= l; }
    c->nfibs[l] = cnt;
    c->fids[l] = malloc((cnt ? cnt : 1) * sizeof(u64));
    c->fptr[l] = (l < nmodes - 1) ? malloc((cnt + 1) * sizeof(u64)) : NULL;
  }
  u64 * cursor = calloc(nmodes, sizeof(u64));
  for(u64 n = 0; n < nnz; ++n) {
    for(u64 l = 0; l < nmodes; ++l) {
      if(l == nmodes - 1 || first[n] <= l) {
        u64 const k = cursor[l]++;
        c->fids[l][k] = lv[l][n];
        if(l < nmodes - 1) {
          /* child index in level l+1 (or nnz position at the last level) */
          c->fptr[l][k] = (l + 1 == nmodes - 1) ? n : cursor[l+1];
        }
      }
    }
  }
  for(u64 l = 0; l + 1 < nmodes; ++l) {
    c->fptr[l][c->nfibs[l]] = c->nfibs[l+1];
  }
  free(cursor);
  free(first);
  free(order);
  for(u64 l = 0; l < nmodes; ++l) { free(lv[l]); }
}

typedef struct { u64 n; orc_csf * t; } orc_set;

/* src/csf.c:695-739 csf_alloc: ONE = SMALLFIRST; TWO = SMALLFIRST plus
 * MINUSONE rooted at the first CSF's leaf mode; ALL = MINUSONE per mode. */
void * orc_csf_alloc(u64 nmodes, u64 nnz, u64 const * dims,
    u64 * const * inds, double const * vals, int alloc_type)
{
  orc_set * s = malloc(sizeof(*s));
  s->n = alloc_type == 0 ? 1 : (alloc_type == 1 ? 2 : nmodes);
  s->t = calloc(s->n, sizeof(orc_csf));
  u64 perm[ORC_MAX_NMODES];
  if(alloc_type == 2) {
    for(u64 m = 0; m < nmodes; ++m) {
      orc_order_minusone(dims, nmodes, m, perm);
      orc_build_one(s->t + m, nmodes, nnz, dims, inds, vals, perm);
    }
  } else {
    orc_order_small(dims, nmodes, perm);
    orc_build_one(s->t, nmodes, nnz, dims, inds, vals, perm);
    if(alloc_type == 1) {
      u64 const leaf = s->t[0].dim_perm[nmodes - 1];
      orc_order_minusone(dims, nmodes, leaf, perm);
      orc_build_one(s->t + 1, nmodes, nnz, dims, inds, vals, perm);
    }
  }
  return s;
}

u64 orc_csf_count(void * h) { return ((orc_set *) h)->n; }
orc_csf const * orc_csf_get(void * h, u64 t) { return ((orc_set *) h)->t + t; }

int orc_csf_info(void * h, u64 t, u64 * nfibs, u64 * dim_perm)
{
  orc_csf const * c = orc_csf_get(h, t);
  for(u64 l = 0; l < c->nmodes; ++l) {
    nfibs[l] = c->nfibs[l];
    dim_perm[l] = c->dim_perm[l];
  }
  return 1;
}

void orc_csf_level(void * h, u64 t, u64 level, u64 * fptr, u64 * fids)
{
  orc_csf const * c = orc_csf_get(h, t);
  if(fptr && level < c->nmodes - 1) {
    memcpy(fptr, c->fptr[level], (c->nfibs[level] + 1) * sizeof(u64));
  }
  if(fids) { memcpy(fids, c->fids[level], c->nfibs[level] * sizeof(u64)); }
}

void orc_csf_vals(void * h, u64 t, double * vals)
{
  orc_csf const * c = orc_csf_get(h, t);
  memcpy(vals, c->vals, c->nnz * sizeof(double));
}

void orc_csf_free(void * h)
{
  orc_set * s = h;
  for(u64 i = 0; i < s->n; ++i) {
    orc_csf * c = s->t + i;
    for(u64 l = 0; l < c->nmodes; ++l) { free(c->fptr[l]); free(c->fids[l]); }
    free(c->vals);
  }
  free(s->t);
  free(s);
}

/* ------------------------------------------------------------------------ */
/* Dense-tiled CSF: src/csf.c:427-501 (p_csf_alloc_densetile) and           */
/* src/tile.c:260-340 (tt_densetile, get_tile_id).  The modes at the        */
/* bottom `tilelevel` levels of a tree are cut into `nthreads` equal index   */
/* ranges (the last one takes the remainder); the nonzeros sorted for the   */
/* tree are stably bucketed by tile id (mode 0 slowest), and every tile is   */
/* its own CSF over its nonzeros, so a tile's order is the tree's sorted    */
/* order restricted to it.  An empty tile has no levels.                    */
/* ------------------------------------------------------------------------ */
/* t[tree * stride + tile]; tree i has nt[i] tiles */
typedef struct { u64 n, stride; u64 nt[ORC_MAX_NMODES]; orc_csf * t; } orc_tset;

static void orc_build_tiled(orc_csf * tiles, u64 * ntiles_out, u64 nmodes, u64 nnz,
    u64 const * dims, u64 * const * inds, double const * vals, u64 const * perm,
    u64 nthreads, u64 tilelevel)
{
  u64 const ntiled = tilelevel < nmodes ? tilelevel : nmodes;
  u64 const depth0 = nmodes - ntiled;
  u64 tdim[ORC_MAX_NMODES], tsize[ORC_MAX_NMODES];
  u64 ntiles = 1;
  for(u64 m = 0; m < nmodes; ++m) {
    u64 depth = 0;
    while(perm[depth] != m) { ++depth; }
    tdim[m] = depth >= depth0 ? nthreads : 1;
    tsize[m] = dims[m] / tdim[m] > 0 ? dims[m] / tdim[m] : 1;
    ntiles *= tdim[m];
  }
  *ntiles_out = ntiles;
  u64 * id = malloc((nnz ? nnz : 1) * sizeof(u64));
  for(u64 n = 0; n < nnz; ++n) {
    u64 x = 0;
    for(u64 m = 0; m < nmodes; ++m) {
      u64 c = inds[m][n] / tsize[m];
      if(c > tdim[m] - 1) { c = tdim[m] - 1; }
      x = x * tdim[m] + c;
    }
    id[n] = x;
  }
  u64 * sub[ORC_MAX_NMODES];
  for(u64 m = 0; m < nmodes; ++m) { sub[m] = malloc((nnz ? nnz : 1) * sizeof(u64)); }
  double * sv = malloc((nnz ? nnz : 1) * sizeof(double));
  for(u64 t = 0; t < ntiles; ++t) {
    u64 k = 0;
    for(u64 n = 0; n < nnz; ++n) {
      if(id[n] != t) { continue; }
      for(u64 m = 0; m < nmodes; ++m) { sub[m][k] = inds[m][n]; }
      sv[k++] = vals[n];
    }
    orc_build_one(tiles + t, nmodes, k, dims, sub, sv, perm);
  }
  for(u64 m = 0; m < nmodes; ++m) { free(sub[m]); }
  free(sv);
  free(id);
}

/* csf_alloc with SPLATT_OPTION_TILE = SPLATT_DENSETILE, SPLATT_OPTION_NTHREADS
 * = nthreads and SPLATT_OPTION_TILELEVEL = tilelevel (src/csf.c:541-558,
 * 695-733: TWOMODE builds its second tree untiled) */
void * orc_csf_alloc_tiled(u64 nmodes, u64 nnz, u64 const * dims,
    u64 * const * inds, double const * vals, int alloc_type, u64 nthreads,
    u64 tilelevel)
{
  orc_tset * s = malloc(sizeof(*s));
  s->n = alloc_type == 0 ? 1 : (alloc_type == 1 ? 2 : nmodes);
  u64 ntiled = tilelevel < nmodes ? tilelevel : nmodes;
  u64 maxt = 1;
  for(u64 i = 0; i < ntiled; ++i) { maxt *= nthreads; }
  s->t = calloc(s->n * maxt, sizeof(orc_csf));
  s->stride = maxt;
  u64 perm[ORC_MAX_NMODES];
  for(u64 i = 0; i < s->n; ++i) {
    if(alloc_type == 2) {
      orc_order_minusone(dims, nmodes, i, perm);
    } else if(i == 0) {
      orc_order_small(dims, nmodes, perm);
    } else {
      orc_order_minusone(dims, nmodes, s->t[0].dim_perm[nmodes - 1], perm);
    }
    u64 const thr = (alloc_type == 1 && i == 1) ? 1 : nthreads;
    orc_build_tiled(s->t + i * maxt, &s->nt[i], nmodes, nnz, dims, inds, vals, perm,
        thr, tilelevel);
  }
  return s;
}

u64 orc_tcsf_count(void * h) { return ((orc_tset *) h)->n; }
u64 orc_tcsf_ntiles(void * h, u64 t) { return ((orc_tset *) h)->nt[t]; }

static orc_csf const * orc_tcsf_get(void * h, u64 t, u64 tile)
{
  orc_tset const * s = h;
  return s->t + t * s->stride + tile;
}

void orc_tcsf_info(void * h, u64 t, u64 tile, u64 * nfibs, u64 * dim_perm)
{
  orc_csf const * c = orc_tcsf_get(h, t, tile);
  for(u64 l = 0; l < c->nmodes; ++l) {
    nfibs[l] = c->nfibs[l];
    dim_perm[l] = c->dim_perm[l];
  }
}

void orc_tcsf_level(void * h, u64 t, u64 tile, u64 level, u64 * fptr, u64 * fids)
{
  orc_csf const * c = orc_tcsf_get(h, t, tile);
  if(fptr && level < c->nmodes - 1) {
    memcpy(fptr, c->fptr[level], (c->nfibs[level] + 1) * sizeof(u64));
  }
  if(fids) { memcpy(fids, c->fids[level], c->nfibs[level] * sizeof(u64)); }
}

void orc_tcsf_vals(void * h, u64 t, u64 tile, double * vals)
{
  orc_csf const * c = orc_tcsf_get(h, t, tile);
  memcpy(vals, c->vals, c->nnz * sizeof(double));
}

void orc_tcsf_free(void * h)
{
  orc_tset * s = h;
  for(u64 i = 0; i < s->n * s->stride; ++i) {
    orc_csf * c = s->t + i;
    if(c->nmodes == 0) { continue; }             /* slot of an untiled tree */
    for(u64 l = 0; l < c->nmodes; ++l) { free(c->fptr[l]); free(c->fids[l]); }
    free(c->vals);
  }
  free(s->t);
  free(s);
}

/* ------------------------------------------------------------------------ */
/* CSF MTTKRP: src/mttkrp.c:390-1278 (root / internal / leaf traversals)    */
/* and the mode->CSF choice of src/mttkrp.c:1831-1880.                      */
/*   S(node at level l) = rows_l[fid] o sum_children S(child)  (l > out)    */
/*   leaf contributes v * rows_leaf[fid]                                     */
/*   out[fid(node at out level)] += prefix o sum_children S(child)          */
/* where prefix = Hadamard of the ancestors' rows (levels < out).            */
/* ------------------------------------------------------------------------ */
static void orc_subtree(orc_csf const * c, double ** mv, u64 level, u64 node,
    u64 R, double * acc, double * tmp)
{
  /* acc += sum over children of `node` (node at `level`) of S(child) */
  u64 const N = c->nmodes;
  u64 const b = c->fptr[level][node];
  u64 const e = c->fptr[level][node+1];
  if(level + 1 == N - 1) {
    double const * B = mv[N-1];
    for(u64 j = b; j < e; ++j) {
      double const v = c->vals[j];
      double const * row = B + c->fids[N-1][j] * R;
      for(u64 r = 0; r < R; ++r) { acc[r] += v * row[r]; }
    }
    return;
  }
  double * child = tmp;
  double * deeper = tmp + R;
  for(u64 k = b; k < e; ++k) {
    for(u64 r = 0; r < R; ++r) { child[r] = 0.; }
    orc_subtree(c, mv, level + 1, k, R, child, deeper);
    double const * row = mv[level+1] + c->fids[level+1][k] * R;
    for(u64 r = 0; r < R; ++r) { acc[r] += row[r] * child[r]; }
  }
}

static void orc_walk(orc_csf const * c, double ** mv, u64 od, u64 level,
    u64 node, double const * prefix, u64 R, double * out, double * scratch)
{
  u64 const N = c->nmodes;
  if(level == od) {
    if(od == N - 1) {                         /* leaf output */
      double const v = c->vals[node];
      double * o = out + c->fids[N-1][node] * R;
      for(u64 r = 0; r < R; ++r) { o[r] += v * prefix[r]; }
      return;
    }
    double * acc = scratch;
    for(u64 r = 0; r < R; ++r) { acc[r] = 0.; }
    orc_subtree(c, mv, level, node, R, acc, scratch + R);
    double * o = out + c->fids[level][node] * R;
    for(u64 r = 0; r < R; ++r) { o[r] += prefix[r] * acc[r]; }
    return;
  }
  /* extend the prefix with this node's row and descend */
  double * np = scratch;
  double const * row = mv[level] + c->fids[level][node] * R;
  for(u64 r = 0; r < R; ++r) { np[r] = prefix[r] * row[r]; }
  u64 const b = c->fptr[level][node];
  u64 const e = c->fptr[level][node+1];
  for(u64 k = b; k < e; ++k) {
    orc_walk(c, mv, od, level + 1, k, np, R, out, scratch + R);
  }
}

void orc_mttkrp(void * h, u64 mode, u64 R, double ** mats, double * out)
{
  orc_set * s = h;
  orc_csf const * c0 = s->t;
  u64 const N = c0->nmodes;
  /* src/mttkrp.c:1849-1880: which CSF serves `mode` */
  orc_csf const * c = c0;
  if(s->n == 2 && c0->dim_perm[N-1] == mode) { c = s->t + 1; }
  if(s->n == N && N > 2) { c = s->t + mode; }
  if(s->n == N && N == 2) { c = s->t + mode; }

  u64 od = 0;
  for(u64 l = 0; l < N; ++l) { if(c->dim_perm[l] == mode) { od = l; } }
  double * mv[ORC_MAX_NMODES];
  for(u64 l = 0; l < N; ++l) { mv[l] = mats[c->dim_perm[l]]; }

  memset(out, 0, c->dims[mode] * R * sizeof(double));
  double * scratch = malloc((2 * N + 4) * R * sizeof(double));
  double * ones = malloc(R * sizeof(double));
  for(u64 r = 0; r < R; ++r) { ones[r] = 1.; }
  for(u64 sl = 0; sl < c->nfibs[0]; ++sl) {
    orc_walk(c, mv, od, 0, sl, ones, R, out, scratch);
  }
  free(ones);
  free(scratch);
}

/* COO MTTKRP: src/mttkrp.c:1699-1769 (mttkrp_stream), one thread. */
void orc_mttkrp_coo(u64 nmodes, u64 nnz, u64 const * dims,
    u64 * const * inds, double const * vals, u64 mode, u64 R,
    double ** mats, double * out)
{
  double * acc = malloc(R * sizeof(double));
  memset(out, 0, dims[mode] * R * sizeof(double));
  for(u64 n = 0; n < nnz; ++n) {
    for(u64 r = 0; r < R; ++r) { acc[r] = vals[n]; }
    for(u64 m = 0; m < nmodes; ++m) {
      if(m == mode) { continue; }
      double const * row = mats[m] + inds[m][n] * R;
      for(u64 r = 0; r < R; ++r) { acc[r] *= row[r]; }
    }
    double * o = out + inds[mode][n] * R;
    for(u64 r = 0; r < R; ++r) { o[r] += acc[r]; }
  }
  free(acc);
}

/* ------------------------------------------------------------------------ */
/* dense kernels: src/matrix.c                                               */
/* Matrices are row-major I x R.  Gram matrices keep the row-major upper     */
/* triangle (= LAPACK's column-major lower) as the reference does.           */
/* ------------------------------------------------------------------------ */

/* mat_aTa (matrix.c:171-205): upper triangle of A^T A */
static void orc_ata(double const * A, u64 I, u64 R, double * G)
{
  for(u64 i = 0; i < R; ++i) {
    for(u64 j = i; j < R; ++j) {
      double s = 0.;
      for(u64 x = 0; x < I; ++x) { s += A[x*R + i] * A[x*R + j]; }
      G[i*R + j] = s;
    }
  }
}

/* mat_form_gram (matrix.c:311-345): Hadamard of all aTa but `mode` (upper) */
static void orc_form_gram(double ** ata, u64 nmodes, u64 mode, u64 R,
    double * G)
{
  for(u64 i = 0; i < R; ++i) {
    for(u64 j = i; j < R; ++j) { G[i*R + j] = 1.; }
  }
  for(u64 m = 0; m < nmodes; ++m) {
    if(m == mode) { continue; }
    for(u64 i = 0; i < R; ++i) {
      for(u64 j = i; j < R; ++j) { G[i*R + j] *= ata[m][i*R + j]; }
    }
  }
}

/* mat_cholesky (matrix.c:104-124): G = L L^T using the row-major upper
 * triangle as L^T; the factor L is stored in place as L[j][i] = G[i*R+j]
 * (i <= j).  Returns the first non-positive pivot + 1, or 0. */
static int orc_cholesky(double * G, u64 R)
{
  for(u64 j = 0; j < R; ++j) {
    double d = G[j*R + j];
    for(u64 k = 0; k < j; ++k) { d -= G[k*R + j] * G[k*R + j]; }
    if(!(d > 0.)) { return (int) j + 1; }
    d = sqrt(d);
    G[j*R + j] = d;
    for(u64 i = j + 1; i < R; ++i) {
      double s = G[j*R + i];
      for(u64 k = 0; k < j; ++k) { s -= G[k*R + j] * G[k*R + i]; }
      G[j*R + i] = s / d;
    }
  }
  return 0;
}

/* mat_solve_cholesky (matrix.c:127-151): every row b of the I x R matrix is
 * replaced by G^{-1} b: forward (L y = b) then backward (L^T x = y). */
static void orc_solve(double const * L, u64 R, double * B, u64 I)
{
  for(u64 x = 0; x < I; ++x) {
    double * b = B + x * R;
    for(u64 i = 0; i < R; ++i) {
      double s = b[i];
      for(u64 k = 0; k < i; ++k) { s -= L[k*R + i] * b[k]; }
      b[i] = s / L[i*R + i];
    }
    for(u64 ii = R; ii-- > 0; ) {
      double s = b[ii];
      for(u64 k = ii + 1; k < R; ++k) { s -= L[ii*R + k] * b[k]; }
      b[ii] = s / L[ii*R + ii];
    }
  }
}

/* mat_normalize / p_mat_2norm (matrix.c:37-96, 277-293) */
static void orc_normalize(double * A, u64 I, u64 R, double * lambda)
{
  for(u64 r = 0; r < R; ++r) { lambda[r] = 0.; }
  for(u64 x = 0; x < I; ++x) {
    for(u64 r = 0; r < R; ++r) { lambda[r] += A[x*R + r] * A[x*R + r]; }
  }
  for(u64 r = 0; r < R; ++r) { lambda[r] = sqrt(lambda[r]); }
  for(u64 x = 0; x < I; ++x) {
    for(u64 r = 0; r < R; ++r) { A[x*R + r] /= lambda[r]; }
  }
}

/* ------------------------------------------------------------------------ */
/* CPD-ALS: src/cpd/cpd.c:116-141 (splatt_alloc_cpd), 161-309 (cpd_iterate),*/
/* 453-531 (cpd_norm, cpd_innerprod); closed-form admm() src/cpd/admm.c:    */
/* 217-235, 316-345.                                                         */
/* ------------------------------------------------------------------------ */
double orc_cpd(u64 nmodes, u64 nnz, u64 const * dims, u64 * const * inds,
    double const * vals, u64 R, u64 niters, double tol, int seed,
    double ** factors, double * lambda, double * fit, double * fit_per_iter)
{
  void * h = orc_csf_alloc(nmodes, nnz, dims, inds, vals, 1);
  orc_csf const * c = orc_csf_get(h, 0);

  srand(seed);
  for(u64 m = 0; m < nmodes; ++m) { orc_fill_rand(factors[m], dims[m] * R); }

  double * ata[ORC_MAX_NMODES];
  for(u64 m = 0; m < nmodes; ++m) { ata[m] = calloc(R * R, sizeof(double)); }
  double * G = malloc(R * R * sizeof(double));
  double * tmpl = malloc(R * sizeof(double));
  u64 maxdim = 0;
  for(u64 m = 0; m < nmodes; ++m) { if(dims[m] > maxdim) { maxdim = dims[m]; } }
  double * M = malloc(maxdim * R * sizeof(double));

  for(u64 m = 0; m < nmodes; ++m) { orc_normalize(factors[m], dims[m], R, lambda); }
  for(u64 r = 0; r < R; ++r) { lambda[r] = 1.; }
  for(u64 m = 1; m < nmodes; ++m) { orc_ata(factors[m], dims[m], R, ata[m]); }

  double xnorm = 0.;
  for(u64 n = 0; n < nnz; ++n) { xnorm += c->vals[n] * c->vals[n]; }

  double olderr = 1., err = 0.;
  u64 it;
  for(it = 0; it < niters; ++it) {
    for(u64 m = 0; m < nmodes; ++m) {
      orc_mttkrp(h, m, R, factors, M);
      orc_form_gram(ata, nmodes, m, R, G);
      orc_cholesky(G, R);
      memcpy(factors[m], M, dims[m] * R * sizeof(double));
      orc_solve(G, R, factors[m], dims[m]);
      orc_normalize(factors[m], dims[m], R, lambda);
      orc_ata(factors[m], dims[m], R, ata[m]);
    }
    /* cpd_norm: lambda^T (Hadamard of all aTa) lambda, upper triangle */
    double norm = 0.;
    for(u64 i = 0; i < R; ++i) {
      for(u64 j = i; j < R; ++j) {
        double g = 1.;
        for(u64 m = 0; m < nmodes; ++m) { g *= ata[m][i*R + j]; }
        norm += (i == j) ? g * lambda[i] * lambda[i]
                         : 2. * g * lambda[i] * lambda[j];
      }
    }
    norm = fabs(norm);
    /* cpd_innerprod with the last mode's MTTKRP */
    u64 const lm = nmodes - 1;
    double inner = 0.;
    for(u64 r = 0; r < R; ++r) {
      double a = 0.;
      for(u64 x = 0; x < dims[lm]; ++x) { a += factors[lm][x*R + r] * M[x*R + r]; }
      inner += a * lambda[r];
    }
    err = (xnorm + norm - 2. * inner) / xnorm;
    if(fit_per_iter) { fit_per_iter[it] = 1. - err; }
    if(it > 0 && fabs(olderr - err) < tol) { ++it; break; }
    olderr = err;
  }
  /* cpd_post_process: absorb column norms into lambda */
  for(u64 m = 0; m < nmodes; ++m) {
    orc_normalize(factors[m], dims[m], R, tmpl);
    for(u64 r = 0; r < R; ++r) { lambda[r] *= tmpl[r]; }
  }
  *fit = 1. - err;

  free(M); free(G); free(tmpl);
  for(u64 m = 0; m < nmodes; ++m) { free(ata[m]); }
  orc_csf_free(h);
  return (double) it;
}

/* ------------------------------------------------------------------------ */
/* Streaming CPD: src/cpd/stream/ParserSimple.cc:13-149 (sort by time,       */
/* first-appearance relabel, slices), src/cpd/stream/StreamCPD.cc:192-571    */
/* (grow_mats, add_historical, compute), src/cpd/admm.c:240-406 (ADMM with   */
/* the max-column-norm prox of src/cpd/constraints/maxcolnorm.c:32-62; with */
/* prox 1 the non-negative one of maxcolnorm-nonneg.c:32-62, which          */
/* StreamCPD.cc:325-337 registers for `--con=nonneg`; with prox 2 lasso in  */
/* 50-row chunks, `--reg=l1,prox_mult`; prox 3 the row simplex, chunked,  */
/* `--con=rowsimp`; prox 4 `--reg=ntf-l1,prox_mult` and prox 5             */
/* `--reg=ntf-frob,prox_mult`, both chunked; prox 6 the column simplex,    */
/* single-chunk, `--con=colsimp`) and                                       */
/* the frob closed form of src/cpd/constraints/frob.c:25-37.                 */
/* ------------------------------------------------------------------------ */

static int orc_desc(void const * a, void const * b)
{
  double const x = *(double const *) a, y = *(double const *) b;
  return x < y ? 1 : (x > y ? -1 : 0);
}

/* projection of one row onto the probability simplex (simplex.cc:34-66):
 * sort a copy descending, find the pivot with a running sum that starts at
 * -1, theta = sum / pivot, x = max(x - theta, 0) */
static void orc_rowsimp(double * x, u64 R, double * buf)
{
  memcpy(buf, x, R * sizeof(double));
  qsort(buf, R, sizeof(double), orc_desc);
  double run = -1.;
  u64 piv;
  for(piv = 0; piv < R; ++piv) {
    run += buf[piv];
    if(buf[piv] - run / (double) (piv + 1) <= 0.) { run -= buf[piv]; break; }
  }
  double const theta = run / (double) piv;
  for(u64 j = 0; j < R; ++j) {
    x[j] -= theta;
    if(x[j] < 0.) { x[j] = 0.; }
  }
}

/* The proximal operators of the ADMM constraints, applied to the I x R
 * row-major block P; `kind` numbers them as orc_stream's `prox` does:
 *   0 max-column-norm: columns with 2-norm > 1 scaled to unit norm
 *     (maxcolnorm.c:32-62);
 *   1 the same after zeroing negatives (maxcolnorm-nonneg.c:32-62);
 *   2 lasso: soft threshold at lambda / rho (lasso.c:29-55);
 *   3 each row onto the probability simplex (simplex.cc:34-66, 82-107);
 *   4 NTF-L1: v > lambda/rho ? v - lambda/rho : 0 (nonneg_lasso.c:29-45);
 *   5 NTF-Frobenius: max(v * rho / (lambda + rho), 0) (nonneg_frob.c:33-49);
 *   6 each column onto the probability simplex (simplex.cc:120-150);
 *   7 non-negativity: negatives zeroed (nonneg.c:31-45).
 * Kinds 2-5 and 7 act on rows independently. */
void orc_prox(int kind, double * P, u64 I, u64 R, double lambda, double rho)
{
  u64 const n = I * R;
  if(kind == 0 || kind == 1) {
    if(kind == 1) {
      for(u64 x = 0; x < n; ++x) { if(P[x] < 0.) { P[x] = 0.; } }
    }
    double * cn = malloc((R ? R : 1) * sizeof(double));
    for(u64 r = 0; r < R; ++r) {
      double s = 0.;
      for(u64 x = 0; x < I; ++x) { s += P[x*R + r] * P[x*R + r]; }
      cn[r] = sqrt(s);
    }
    for(u64 x = 0; x < I; ++x) {
      for(u64 r = 0; r < R; ++r) {
        if(cn[r] > 1.) { P[x*R + r] /= cn[r]; }
      }
    }
    free(cn);
  } else if(kind == 2) {
    double const mult = lambda / rho;
    for(u64 x = 0; x < n; ++x) {
      double const v = P[x];
      P[x] = v > mult ? v - mult : (v < -mult ? v + mult : 0.);
    }
  } else if(kind == 3) {
    double * buf = malloc((R ? R : 1) * sizeof(double));
    for(u64 r = 0; r < I; ++r) { orc_rowsimp(P + r * R, R, buf); }
    free(buf);
  } else if(kind == 4) {
    double const mult = lambda / rho;
    for(u64 x = 0; x < n; ++x) { P[x] = P[x] > mult ? P[x] - mult : 0.; }
  } else if(kind == 5) {
    double const shrink = rho / (lambda + rho);
    for(u64 x = 0; x < n; ++x) {
      double const v = P[x] * shrink;
      P[x] = v > 0. ? v : 0.;
    }
  } else if(kind == 6) {
    double * col = malloc((I ? I : 1) * sizeof(double));
    double * buf = malloc((I ? I : 1) * sizeof(double));
    for(u64 r = 0; r < R; ++r) {
      for(u64 x = 0; x < I; ++x) { col[x] = P[x*R + r]; }
      orc_rowsimp(col, I, buf);
      for(u64 x = 0; x < I; ++x) { P[x*R + r] = col[x]; }
    }
    free(buf);
    free(col);
  } else if(kind == 7) {
    for(u64 x = 0; x < n; ++x) { if(P[x] < 0.) { P[x] = 0.; } }
  }
}

/* One ADMM solve (src/cpd/admm.c:240-308) on rows [c0, c1) of the I x R
 * primal P, with the prox `kind` of orc_prox: iterate aux = (M + rho (P + D))
 * L^-T L^-1, P = prox(aux - D), D += P - aux until the residual test passes.
 * Returns the iterations taken. */
static u64 orc_admm_block(double * P, double * aux, double * D, double * init,
    double const * Mk, double const * L, double rho, u64 c0, u64 c1, u64 R,
    u64 max_inner, double inner_tol, int kind, double lambda)
{
  u64 const b = c0 * R, e = c1 * R;
  u64 it;
  for(it = 0; it < max_inner; ++it) {
    memcpy(init + b, P + b, (e - b) * sizeof(double));
    for(u64 x = b; x < e; ++x) { aux[x] = Mk[x] + rho * (P[x] + D[x]); }
    orc_solve(L, R, aux + b, c1 - c0);
    for(u64 x = b; x < e; ++x) { P[x] = aux[x] - D[x]; }
    orc_prox(kind, P + b, c1 - c0, R, lambda, rho);
    double dnorm = 0., pnorm = 0., presid = 0., dresid = 0.;
    for(u64 x = b; x < e; ++x) {
      D[x] += P[x] - aux[x];
      dnorm += D[x] * D[x];
    }
    for(u64 x = b; x < e; ++x) {
      double const pd = P[x] - aux[x];
      double const dd = P[x] - init[x];
      pnorm += P[x] * P[x];
      presid += pd * pd;
      dresid += dd * dd;
    }
    if(presid <= inner_tol * pnorm && dresid <= inner_tol * dnorm) { ++it; break; }
  }
  return it;
}

/* src/cpd/admm.c:352-395: a row-separable prox (kinds 2-5) runs in
 * independent chunks of `chunk` rows, each to its own residual test, and
 * reports iterations x rows summed over chunks; any other runs as one chunk
 * and reports its iterations. */
static u64 orc_admm(double * P, double * aux, double * D, double * init,
    double const * Mk, double const * L, double rho, u64 I, u64 R,
    u64 max_inner, double inner_tol, int kind, double lambda, u64 chunk)
{
  if(kind < 2 || kind > 5) {
    return orc_admm_block(P, aux, D, init, Mk, L, rho, 0, I, R, max_inner, inner_tol,
        kind, lambda);
  }
  u64 total = 0;
  for(u64 c0 = 0; c0 < I; c0 += chunk) {
    u64 const c1 = c0 + chunk < I ? c0 + chunk : I;
    total += orc_admm_block(P, aux, D, init, Mk, L, rho, c0, c1, R, max_inner, inner_tol,
        kind, lambda) * (c1 - c0);
  }
  return total;
}

/* lexicographic order with `first` leading and the rest rotating after it,
 * the default tie-breaking of src/sort.c:921-956 when dim_perm is NULL */
static u64 * orc_stream_order(u64 nmodes, u64 nnz, u64 * const * inds, u64 sm)
{
  u64 perm[ORC_MAX_NMODES];
  for(u64 m = 0; m < nmodes; ++m) { perm[m] = (sm + m) % nmodes; }
  return orc_sorted_order(nmodes, nnz, inds, perm);
}

/* ParserSimple's constructor (src/cpd/stream/ParserSimple.cc:13-79): sort
 * by time, relabel every other mode by first appearance in that order.
 * sind[m] and *sval are malloc'd here and owned by the caller. */
static void orc_stream_parse(u64 nmodes, u64 nnz, u64 const * dims,
    u64 * const * inds, double const * vals, u64 sm, u64 ** sind, double ** sval)
{
  u64 * order = orc_stream_order(nmodes, nnz, inds, sm);
  *sval = malloc((nnz ? nnz : 1) * sizeof(double));
  for(u64 m = 0; m < nmodes; ++m) {
    sind[m] = malloc((nnz ? nnz : 1) * sizeof(u64));
    for(u64 n = 0; n < nnz; ++n) { sind[m][n] = inds[m][order[n]]; }
  }
  for(u64 n = 0; n < nnz; ++n) { (*sval)[n] = vals[order[n]]; }
  free(order);
  for(u64 m = 0; m < nmodes; ++m) {
    if(m == sm) { continue; }
    u64 * lab = malloc(dims[m] * sizeof(u64));
    for(u64 i = 0; i < dims[m]; ++i) { lab[i] = UINT64_MAX; }
    u64 seen = 0;
    for(u64 n = 0; n < nnz; ++n) {
      u64 const x = sind[m][n];
      if(lab[x] == UINT64_MAX) { lab[x] = seen++; }
      sind[m][n] = lab[x];
    }
    free(lab);
  }
}

/* the parser's preparation alone, into caller arrays of nnz entries each */
void orc_stream_prepare(u64 nmodes, u64 nnz, u64 const * dims, u64 * const * inds,
    double const * vals, u64 sm, u64 * const * out_inds, double * out_vals)
{
  u64 * sind[ORC_MAX_NMODES];
  double * sval = NULL;
  orc_stream_parse(nmodes, nnz, dims, inds, vals, sm, sind, &sval);
  for(u64 m = 0; m < nmodes; ++m) {
    memcpy(out_inds[m], sind[m], nnz * sizeof(u64));
    free(sind[m]);
  }
  memcpy(out_vals, sval, nnz * sizeof(double));
  free(sval);
}

u64 orc_stream(u64 nmodes, u64 nnz, u64 const * dims, u64 * const * inds,
    double const * vals, u64 sm, u64 R, double forget, double reg,
    u64 max_its, int seed, u64 max_slices, double * time_out,
    double ** factors, u64 * out_rows, u64 * outer_its, double * local_errsq, int prox,
    double prox_mult)
{
  /* --- ParserSimple: sort by time, relabel other modes by first use --- */
  u64 * sind[ORC_MAX_NMODES];
  double * sval = NULL;
  orc_stream_parse(nmodes, nnz, dims, inds, vals, sm, sind, &sval);

  /* --- state (StreamCPD members) --- */
  u64 cap[ORC_MAX_NMODES];
  for(u64 m = 0; m < nmodes; ++m) { cap[m] = dims[m] > 0 ? dims[m] : 1; }
  u64 maxcap = 1;
  for(u64 m = 0; m < nmodes; ++m) { if(m != sm && cap[m] > maxcap) { maxcap = cap[m]; } }
  double * anew[ORC_MAX_NMODES], * aold[ORC_MAX_NMODES], * dual[ORC_MAX_NMODES];
  double * ata[ORC_MAX_NMODES];
  u64 rows[ORC_MAX_NMODES];
  for(u64 m = 0; m < nmodes; ++m) {
    anew[m] = calloc(cap[m] * R, sizeof(double));
    aold[m] = calloc(cap[m] * R, sizeof(double));
    dual[m] = calloc(cap[m] * R, sizeof(double));
    ata[m] = calloc(R * R, sizeof(double));
    rows[m] = 0;
  }
  double * Mbuf = calloc(maxcap * R, sizeof(double));
  double * aux = calloc(maxcap * R, sizeof(double));
  double * init = calloc(maxcap * R, sizeof(double));
  double * G = malloc(R * R * sizeof(double));
  double * oldgram = calloc(R * R, sizeof(double));
  double * hbuf = malloc(R * R * sizeof(double));
  double * hist = malloc(R * R * sizeof(double));
  double * s = calloc(R, sizeof(double));
  double * lam = malloc(R * sizeof(double));
  u64 sdims[ORC_MAX_NMODES];
  u64 prevdim[ORC_MAX_NMODES] = {0};
  u64 * bind[ORC_MAX_NMODES];

  srand(seed);
  u64 ptr = 0, t = 0;
  while(ptr < nnz && (max_slices == 0 || t < max_slices)) {
    /* --- next_batch: the nonzeros whose time index equals t --- */
    u64 start = ptr;
    while(start < nnz && sind[sm][start] < t) { ++start; }
    u64 end = start;
    while(end < nnz && sind[sm][end] < t + 1) { ++end; }
    u64 const bn = end - start;
    for(u64 m = 0; m < nmodes; ++m) {
      bind[m] = sind[m] + start;
      if(m == sm) { sdims[m] = 1; continue; }
      u64 mx = 0;
      for(u64 n = 0; n < bn; ++n) { if(bind[m][n] > mx) { mx = bind[m][n]; } }
      sdims[m] = (mx + 1 > prevdim[m]) ? mx + 1 : prevdim[m];
      prevdim[m] = sdims[m];
    }
    /* time-mode indices inside a batch are all zero */
    u64 * zeros = calloc(bn ? bn : 1, sizeof(u64));
    u64 * bptr[ORC_MAX_NMODES];
    for(u64 m = 0; m < nmodes; ++m) { bptr[m] = (m == sm) ? zeros : bind[m]; }
    double const * bval = sval + start;

    /* --- grow_mats: new rows random (mode order), Gram of new factors --- */
    for(u64 m = 0; m < nmodes; ++m) {
      if(m == sm) { continue; }
      if(sdims[m] > rows[m]) {
        orc_fill_rand(anew[m] + rows[m] * R, (sdims[m] - rows[m]) * R);
        rows[m] = sdims[m];
      }
      orc_ata(anew[m], rows[m], R, ata[m]);
    }
    if(t == 0) {
      for(u64 m = 0; m < nmodes; ++m) {
        if(m != sm) { orc_normalize(anew[m], rows[m], R, lam); }
      }
    }

    double * mats[ORC_MAX_NMODES];
    for(u64 m = 0; m < nmodes; ++m) { mats[m] = (m == sm) ? s : anew[m]; }
    u64 mdims[ORC_MAX_NMODES];
    for(u64 m = 0; m < nmodes; ++m) { mdims[m] = (m == sm) ? 1 : rows[m]; }

    double prev_delta = 0.;
    u64 outer;
    for(outer = 0; outer < max_its; ++outer) {
      double delta = 0.;
      /* time row: MTTKRP + frob closed form */
      orc_mttkrp_coo(nmodes, bn, mdims, bptr, bval, sm, R, mats, Mbuf);
      orc_form_gram(ata, nmodes, sm, R, G);
      for(u64 r = 0; r < R; ++r) { G[r*R + r] += reg; }
      orc_cholesky(G, R);
      memcpy(s, Mbuf, R * sizeof(double));
      orc_solve(G, R, s, 1);

      /* temporal Gram: mirror upper to lower, save, add s s^T */
      for(u64 i = 1; i < R; ++i) {
        for(u64 j = 0; j < i; ++j) { ata[sm][i*R + j] = ata[sm][j*R + i]; }
      }
      memcpy(oldgram, ata[sm], R * R * sizeof(double));
      for(u64 i = 0; i < R; ++i) {
        for(u64 j = 0; j < R; ++j) { ata[sm][i*R + j] += s[i] * s[j]; }
      }

      for(u64 m = 0; m < nmodes; ++m) {
        if(m == sm) { continue; }
        u64 const I = rows[m];
        orc_mttkrp_coo(nmodes, bn, mdims, bptr, bval, m, R, mats, Mbuf);

        /* add_historical */
        memcpy(hbuf, oldgram, R * R * sizeof(double));
        for(u64 i = 1; i < R; ++i) {
          for(u64 j = 0; j < i; ++j) { hbuf[i*R + j] = hbuf[j*R + i]; }
        }
        for(u64 o = 0; o < nmodes; ++o) {
          if(o == m || o == sm) { continue; }
          for(u64 i = 0; i < R; ++i) {
            for(u64 j = 0; j < R; ++j) {
              double acc = 0.;
              for(u64 x = 0; x < rows[o]; ++x) { acc += aold[o][x*R + i] * anew[o][x*R + j]; }
              hist[i*R + j] = acc;
            }
          }
          for(u64 x = 0; x < R * R; ++x) { hbuf[x] *= hist[x]; }
        }
        for(u64 x = 0; x < I; ++x) {
          for(u64 j = 0; j < R; ++j) {
            double acc = 0.;
            for(u64 k = 0; k < R; ++k) { acc += aold[m][x*R + k] * hbuf[k*R + j]; }
            Mbuf[x*R + j] += acc;
          }
        }

        memset(dual[m], 0, I * R * sizeof(double));
        orc_form_gram(ata, nmodes, m, R, G);
        double tr = 0.;
        for(u64 r = 0; r < R; ++r) { tr += G[r*R + r]; }
        double const rho = tr / (double) R;
        for(u64 r = 0; r < R; ++r) { G[r*R + r] += rho; }
        orc_cholesky(G, R);
        orc_admm(anew[m], aux, dual[m], init, Mbuf, G, rho, I, R, 25, 7e-2, prox, prox_mult, 50);
        orc_ata(anew[m], I, R, ata[m]);

        double nd = 0., nn = 0.;
        for(u64 x = 0; x < I * R; ++x) {
          double const d = aold[m][x] - anew[m][x];
          nd += d * d;
          nn += anew[m][x] * anew[m][x];
        }
        delta += sqrt(nd) / sqrt(nn);
      }
      if(outer > 0 && fabs(delta - prev_delta) < 5e-2) { ++outer; break; }
      prev_delta = delta;
    }
    if(outer_its) { outer_its[t] = outer; }

    for(u64 x = 0; x < R * R; ++x) { ata[sm][x] *= forget; }
    for(u64 m = 0; m < nmodes; ++m) {
      if(m != sm) { memcpy(aold[m], anew[m], rows[m] * R * sizeof(double)); }
    }
    memcpy(time_out + t * R, s, R * sizeof(double));

    /* per-slice error on the latest slice (StreamCPD.cc:77-86 ->
     * cpd.c:580-656); lambda = 1, MTTKRP on the smallest mode */
    if(local_errsq) {
      u64 small = 0;
      for(u64 m = 1; m < nmodes; ++m) { if(mdims[m] < mdims[small]) { small = m; } }
      orc_mttkrp_coo(nmodes, bn, mdims, bptr, bval, small, R, mats, Mbuf);
      double inner = 0.;
      for(u64 r = 0; r < R; ++r) {
        double a = 0.;
        for(u64 x = 0; x < mdims[small]; ++x) { a += mats[small][x*R + r] * Mbuf[x*R + r]; }
        inner += a;
      }
      double xn = 0.;
      for(u64 n = 0; n < bn; ++n) { xn += bval[n] * bval[n]; }
      double zn = 0.;
      for(u64 i = 0; i < R; ++i) {
        for(u64 j = i; j < R; ++j) {
          double g = 1.;
          for(u64 m = 0; m < nmodes; ++m) {
            double a = 0.;
            for(u64 x = 0; x < mdims[m]; ++x) { a += mats[m][x*R + i] * mats[m][x*R + j]; }
            g *= a;
          }
          zn += (i == j) ? g : 2. * g;
        }
      }
      zn = fabs(zn);
      double const e = sqrt(xn + zn - 2. * inner) / sqrt(xn);
      local_errsq[t] = e * e;
    }

    free(zeros);
    ptr = end;
    ++t;
  }

  for(u64 m = 0; m < nmodes; ++m) {
    out_rows[m] = (m == sm) ? t : rows[m];
    if(m != sm && factors && factors[m]) {
      memcpy(factors[m], anew[m], rows[m] * R * sizeof(double));
    }
    free(anew[m]); free(aold[m]); free(dual[m]); free(ata[m]); free(sind[m]);
  }
  free(sval); free(Mbuf); free(aux); free(init); free(G); free(oldgram);
  free(hbuf); free(hist); free(s); free(lam);
  return t;
}

/*
 * The streaming driver's windowed error (StreamCPD::compute_errorsq,
 * src/cpd/stream/StreamCPD.cc:77-86) after `nslices` slices: the nonzeros of
 * the last k slices (ParserSimple::stream_prev, ParserSimple.cc:185-226, on
 * the relabeled time-sorted tensor) against the Kruskal tensor of lambda = 1,
 * the last min(k, nslices) time rows and the current factors
 * (StreamCPD::get_prev_kruskal, StreamCPD.cc:150-186), by cpd_error
 * (src/cpd/cpd.c:580-656):
 *   err^2 = (||X||^2 + ||Z||^2 - 2 <X, Z>) / ||X||^2.
 * The inner product is formed as cpd_error forms it: an MTTKRP into the
 * smallest mode of the window, then the dot with that mode's factor.
 * k = nslices gives the report's "global" term, k = 10 "local-10" and, over a
 * completed stream, k = nslices is also "final-err" (StreamCPD.cc:553-556).
 * time_rows: nslices x R; factors[m] (m != sm): rows[m] x R in relabeled
 * order.  Returns -1 when the window holds no nonzeros.
 */
double orc_stream_window_errsq(u64 nmodes, u64 nnz, u64 const * dims,
    u64 * const * inds, double const * vals, u64 sm, u64 R, u64 nslices,
    double const * time_rows, double * const * factors, u64 const * rows, u64 k)
{
  u64 * sind[ORC_MAX_NMODES];
  double * sval = NULL;
  orc_stream_parse(nmodes, nnz, dims, inds, vals, sm, sind, &sval);
  u64 const nk = k < nslices ? k : nslices;
  u64 const start_time = nslices - nk;
  u64 lo = 0;
  while(lo < nnz && sind[sm][lo] < start_time) { ++lo; }
  u64 hi = lo;
  while(hi < nnz && sind[sm][hi] < nslices) { ++hi; }
  u64 const wn = hi - lo;
  double errsq = -1.;
  if(wn > 0 && nk > 0) {
    u64 wdims[ORC_MAX_NMODES];
    u64 * wind[ORC_MAX_NMODES];
    double * mats[ORC_MAX_NMODES];
    u64 * tshift = malloc(wn * sizeof(u64));
    for(u64 n = 0; n < wn; ++n) { tshift[n] = sind[sm][lo + n] - start_time; }
    for(u64 m = 0; m < nmodes; ++m) {
      if(m == sm) {
        wdims[m] = nk;
        wind[m] = tshift;
        mats[m] = (double *) time_rows + start_time * R;
      } else {
        wdims[m] = rows[m];
        wind[m] = sind[m] + lo;
        mats[m] = factors[m];
      }
    }
    u64 small = 0;
    for(u64 m = 1; m < nmodes; ++m) { if(wdims[m] < wdims[small]) { small = m; } }
    double * M = calloc(wdims[small] * R, sizeof(double));
    orc_mttkrp_coo(nmodes, wn, wdims, wind, sval + lo, small, R, mats, M);
    double inner = 0.;
    for(u64 r = 0; r < R; ++r) {
      double a = 0.;
      for(u64 x = 0; x < wdims[small]; ++x) { a += mats[small][x*R + r] * M[x*R + r]; }
      inner += a;
    }
    double xn = 0.;
    for(u64 n = 0; n < wn; ++n) { xn += sval[lo + n] * sval[lo + n]; }
    double zn = 0.;
    for(u64 i = 0; i < R; ++i) {
      for(u64 j = i; j < R; ++j) {
        double g = 1.;
        for(u64 m = 0; m < nmodes; ++m) {
          double a = 0.;
          for(u64 x = 0; x < wdims[m]; ++x) { a += mats[m][x*R + i] * mats[m][x*R + j]; }
          g *= a;
        }
        zn += (i == j) ? g : 2. * g;
      }
    }
    zn = fabs(zn);
    double const e = sqrt(xn + zn - 2. * inner) / sqrt(xn);
    errsq = e * e;
    free(M);
    free(tshift);
  }
  for(u64 m = 0; m < nmodes; ++m) { free(sind[m]); }
  free(sval);
  return errsq;
}
