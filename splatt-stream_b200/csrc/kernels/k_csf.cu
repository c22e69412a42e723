/*
 * k_csf.cu -- CSF construction on the device.
 *
 * Replaces the reference's p_csf_alloc_untiled / p_mk_outerptr / p_mk_fptr
 * (src/csf.c:230-416) and its tt_sort (src/sort.c:761-956):
 *   1. lexicographic order under dim_perm: stable LSD radix sort of a
 *      permutation, one mode at a time from the leaf level up;
 *   2. gather every level's coordinates and the values into that order;
 *   3. for each nonzero, the first level at which its coordinate prefix
 *      differs from its predecessor's ("first-diff level");
 *   4. per level l < N-1: node starts = positions whose first-diff <= l;
 *      exclusive scan numbers them; fids[l] = coordinate at the start,
 *      fptr[l] = index of the first child (position in level l+1, or the
 *      nonzero position at level N-2).
 * The arrays are bit-identical to the reference's for distinct coordinates.
 */
#include "common.cuh"

namespace sb {

__global__ void k_iota(uint32_t * p, uint64_t n)
{
  uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(i < n) { p[i] = (uint32_t) i; }
}

__global__ void k_gather_u32(uint32_t const * __restrict__ src,
    uint32_t const * __restrict__ perm, uint32_t * __restrict__ dst, uint64_t n)
{
  uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(i < n) { dst[i] = __ldg(src + perm[i]); }
}

template <typename T>
__global__ void k_gather_val(T const * __restrict__ src,
    uint32_t const * __restrict__ perm, T * __restrict__ dst, uint64_t n)
{
  uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(i < n) { dst[i] = __ldg(src + perm[i]); }
}

/* first level at which position i's coordinate differs from position i-1 */
struct LevelPtrs { uint32_t const * lv[SB_MAX_NMODES]; };

__global__ void k_first_diff(LevelPtrs L, uint32_t nmodes, uint64_t n,
    uint8_t * __restrict__ fd)
{
  uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n) { return; }
  uint32_t l = 0;
  if(i > 0) {
    while(l + 1 < nmodes && L.lv[l][i] == L.lv[l][i-1]) { ++l; }
  }
  fd[i] = (uint8_t) l;
}

__global__ void k_level_flags(uint8_t const * __restrict__ fd, uint32_t level,
    uint64_t n, uint32_t * __restrict__ flag)
{
  uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(i < n) { flag[i] = fd[i] <= level ? 1u : 0u; }
}

/* scatter node data of level `level` */
__global__ void k_level_scatter(uint8_t const * __restrict__ fd, uint32_t level,
    uint64_t n, uint32_t const * __restrict__ pos, uint32_t const * __restrict__ child_pos,
    uint32_t const * __restrict__ coord, uint32_t * __restrict__ fptr,
    uint32_t * __restrict__ fids)
{
  uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n || fd[i] > level) { return; }
  uint32_t const k = pos[i];
  fids[k] = coord[i];
  fptr[k] = child_pos ? child_pos[i] : (uint32_t) i;
}

__global__ void k_set_u32(uint32_t * p, uint32_t v) { *p = v; }

__global__ void k_narrow(uint64_t const * __restrict__ src, uint32_t * __restrict__ dst,
    uint64_t n, uint64_t dim, int * __restrict__ bad)
{
  uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n) { return; }
  uint64_t const x = src[i];
  if(x >= dim) { *bad = 1; }
  dst[i] = (uint32_t) x;
}

__global__ void k_check(uint32_t const * __restrict__ src, uint64_t n, uint64_t dim,
    int * __restrict__ bad)
{
  uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(i < n && src[i] >= dim) { *bad = 1; }
}

template <typename T>
__global__ void k_frobsq(T const * __restrict__ v, uint64_t n, double * out)
{
  double s = 0.;
  for(uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += (uint64_t) gridDim.x * blockDim.x) {
    double x = (double) v[i];
    s += x * x;
  }
  s = warp_sum(s);
  if((threadIdx.x & 31) == 0) { atomicAdd(out, s); }
}

/* dense-tile id of every nonzero (src/tile.c:260-340): per mode the index
 * range is cut into tdim[m] pieces of tsize[m] (the last takes the rest);
 * mode 0 varies slowest */
struct TileGeom {
  uint32_t const * inds[SB_MAX_NMODES];
  uint64_t tsize[SB_MAX_NMODES];
  uint32_t tdim[SB_MAX_NMODES];
  uint32_t nmodes;
};

__global__ void k_tile_id(TileGeom const g, uint64_t n, uint32_t * __restrict__ id,
    uint32_t * __restrict__ counts)
{
  for(uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += (uint64_t) gridDim.x * blockDim.x) {
    uint64_t x = 0;
    for(uint32_t m = 0; m < g.nmodes; ++m) {
      uint64_t c = (uint64_t) __ldg(g.inds[m] + i) / g.tsize[m];
      if(c > g.tdim[m] - 1) { c = g.tdim[m] - 1; }
      x = x * g.tdim[m] + c;
    }
    id[i] = (uint32_t) x;
    atomicAdd(counts + x, 1u);
  }
}

template <typename S, typename D>
__global__ void k_convert(S const * __restrict__ s, D * __restrict__ d, uint64_t n)
{
  uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(i < n) { d[i] = (D) s[i]; }
}

static int ceil_log2(uint64_t x)
{
  int b = 0;
  while(b < 64 && (1ull << b) < x) { ++b; }
  return b;
}

static void release(sb_dcsf * c)
{
  for(int l = 0; l < SB_MAX_NMODES; ++l) {
    if(c->fptr[l]) { cudaFreeAsync(c->fptr[l], stream()); c->fptr[l] = nullptr; }
    if(c->fids[l]) { cudaFreeAsync(c->fids[l], stream()); c->fids[l] = nullptr; }
  }
  if(c->vals) { cudaFreeAsync(c->vals, stream()); c->vals = nullptr; }
}

} /* namespace sb */

using namespace sb;

extern "C" {

void sb_csf_release(sb_dcsf * c) { release(c); }

int sb_narrow_u64(uint64_t const * src, uint32_t * dst, uint64_t n, uint64_t dim)
{
  if(n == 0) { return SB_OK; }
  int * bad = nullptr;
  int rc = talloc(&bad, 1);
  if(rc) { return rc; }
  SB_TRY(cudaMemsetAsync(bad, 0, sizeof(int), stream()));
  k_narrow<<<blocks_for(n, 256), 256, 0, stream()>>>(src, dst, n, dim, bad);
  SB_CHECK_LAUNCH();
  int h = 0;
  SB_TRY(cudaMemcpyAsync(&h, bad, sizeof(int), cudaMemcpyDeviceToHost, stream()));
  SB_TRY(cudaStreamSynchronize(stream()));
  tfree(bad);
  return h ? SB_EINPUT : SB_OK;
}

int sb_check_u32(uint32_t const * src, uint64_t n, uint64_t dim)
{
  if(n == 0) { return SB_OK; }
  int * bad = nullptr;
  int rc = talloc(&bad, 1);
  if(rc) { return rc; }
  SB_TRY(cudaMemsetAsync(bad, 0, sizeof(int), stream()));
  k_check<<<blocks_for(n, 256), 256, 0, stream()>>>(src, n, dim, bad);
  SB_CHECK_LAUNCH();
  int h = 0;
  SB_TRY(cudaMemcpyAsync(&h, bad, sizeof(int), cudaMemcpyDeviceToHost, stream()));
  SB_TRY(cudaStreamSynchronize(stream()));
  tfree(bad);
  return h ? SB_EINPUT : SB_OK;
}

int sb_frobsq(void const * vals, int vt, uint64_t n, double * out)
{
  double * d = nullptr;
  int rc = talloc(&d, 1);
  if(rc) { return rc; }
  SB_TRY(cudaMemsetAsync(d, 0, sizeof(double), stream()));
  unsigned const g = (unsigned) (n / 256 + 1 < 148 * 8 ? n / 256 + 1 : 148 * 8);
  if(n) {
    if(vt == SB_F64) {
      k_frobsq<double><<<g, 256, 0, stream()>>>((double const *) vals, n, d);
    } else {
      k_frobsq<float><<<g, 256, 0, stream()>>>((float const *) vals, n, d);
    }
    SB_CHECK_LAUNCH();
  }
  SB_TRY(cudaMemcpyAsync(out, d, sizeof(double), cudaMemcpyDeviceToHost, stream()));
  SB_TRY(cudaStreamSynchronize(stream()));
  tfree(d);
  return SB_OK;
}

int sb_convert_vals(void const * src, int st, void * dst, int dt, uint64_t n)
{
  if(n == 0) { return SB_OK; }
  unsigned const b = blocks_for(n, 256);
  if(st == dt) {
    SB_TRY(cudaMemcpyAsync(dst, src, n * (st == SB_F64 ? 8 : 4), cudaMemcpyDeviceToDevice, stream()));
  } else if(st == SB_F64) {
    k_convert<double, float><<<b, 256, 0, stream()>>>((double const *) src, (float *) dst, n);
  } else {
    k_convert<float, double><<<b, 256, 0, stream()>>>((float const *) src, (double *) dst, n);
  }
  SB_CHECK_LAUNCH();
  return SB_OK;
}

int sb_csf_build(uint32_t nmodes, uint64_t nnz, uint64_t const * dims,
    uint32_t * const * inds, void const * vals, int vt,
    uint32_t const * dim_perm, sb_dcsf * out)
{
  memset(out, 0, sizeof(*out));
  if(nmodes < 2 || nmodes > SB_MAX_NMODES || nnz == 0 || nnz >= 0xffffffffull) {
    return SB_EINPUT;
  }
  out->nmodes = nmodes;
  out->nnz = nnz;
  out->val_type = vt;
  for(uint32_t m = 0; m < nmodes; ++m) {
    out->dims[m] = dims[m];
    out->dim_perm[m] = dim_perm[m];
  }
  size_t const vbytes = vt == SB_F64 ? 8 : 4;
  unsigned const nb = blocks_for(nnz, 256);
  cudaStream_t s = stream();

  uint32_t * perm = nullptr, * keys = nullptr, * perm2 = nullptr, * keys2 = nullptr;
  uint32_t * lv[SB_MAX_NMODES] = {nullptr};
  uint8_t * fd = nullptr;
  uint32_t * flag = nullptr, * pos = nullptr, * pos_child = nullptr;
  int rc = SB_OK;

#define SB_STEP(x) do { rc = (x); if(rc) { goto done; } } while(0)
  SB_STEP(talloc(&perm, nnz));
  SB_STEP(talloc(&keys, nnz));
  SB_STEP(talloc(&perm2, nnz));
  SB_STEP(talloc(&keys2, nnz));
  k_iota<<<nb, 256, 0, s>>>(perm, nnz);

  /* 1. LSD over levels, leaf first */
  for(int l = (int) nmodes - 1; l >= 0; --l) {
    uint32_t const m = dim_perm[l];
    int const bits = ceil_log2(dims[m]);
    if(bits == 0) { continue; }
    k_gather_u32<<<nb, 256, 0, s>>>(inds[m], perm, keys, nnz);
    int alt = 0;
    SB_STEP(sb_radix_sort_pairs(keys, perm, keys2, perm2, nnz, bits, &alt));
    if(alt) {
      uint32_t * t = perm; perm = perm2; perm2 = t;
      t = keys; keys = keys2; keys2 = t;
    }
  }

  /* 2. level coordinates + values in sorted order */
  for(uint32_t l = 0; l < nmodes; ++l) {
    SB_STEP(talloc(&lv[l], nnz));
    k_gather_u32<<<nb, 256, 0, s>>>(inds[dim_perm[l]], perm, lv[l], nnz);
  }
  SB_TRY(cudaMallocAsync(&out->vals, nnz * vbytes, s));
  if(vt == SB_F64) {
    k_gather_val<double><<<nb, 256, 0, s>>>((double const *) vals, perm, (double *) out->vals, nnz);
  } else {
    k_gather_val<float><<<nb, 256, 0, s>>>((float const *) vals, perm, (float *) out->vals, nnz);
  }
  out->fids[nmodes-1] = lv[nmodes-1];
  lv[nmodes-1] = nullptr;
  out->nfibs[nmodes-1] = nnz;

  /* 3. first-diff level */
  {
    LevelPtrs L;
    for(uint32_t l = 0; l < SB_MAX_NMODES; ++l) {
      L.lv[l] = l < nmodes - 1 ? lv[l] : out->fids[nmodes-1];
    }
    SB_STEP(talloc(&fd, nnz));
    k_first_diff<<<nb, 256, 0, s>>>(L, nmodes, nnz, fd);
  }

  /* 4. levels N-2 .. 0 */
  SB_STEP(talloc(&flag, nnz));
  SB_STEP(talloc(&pos, nnz));
  SB_STEP(talloc(&pos_child, nnz));
  for(int l = (int) nmodes - 2; l >= 0; --l) {
    k_level_flags<<<nb, 256, 0, s>>>(fd, (uint32_t) l, nnz, flag);
    uint64_t nf = 0;
    SB_STEP(sb_exclusive_scan_u32(flag, pos, nnz, &nf));
    out->nfibs[l] = nf;
    SB_TRY(cudaMallocAsync(&out->fids[l], nf * 4, s));
    SB_TRY(cudaMallocAsync(&out->fptr[l], (nf + 1) * 4, s));
    bool const last = (l == (int) nmodes - 2);
    k_level_scatter<<<nb, 256, 0, s>>>(fd, (uint32_t) l, nnz, pos,
        last ? nullptr : pos_child, lv[l], out->fptr[l], out->fids[l]);
    uint32_t const endv = last ? (uint32_t) nnz : (uint32_t) out->nfibs[l+1];
    k_set_u32<<<1, 1, 0, s>>>(out->fptr[l] + nf, endv);
    uint32_t * t = pos; pos = pos_child; pos_child = t;
  }
  SB_CHECK_LAUNCH();

done:
#undef SB_STEP
  tfree(perm); tfree(keys); tfree(perm2); tfree(keys2);
  for(uint32_t l = 0; l < nmodes; ++l) { tfree(lv[l]); }
  tfree(fd); tfree(flag); tfree(pos); tfree(pos_child);
  if(rc) { release(out); }
  return rc;
}

/* Dense tiling: partition a COO by tile id (the bucket pass of tt_densetile,
 * src/tile.c:260-322).  inds_out / vals_out receive the nonzeros grouped by
 * tile in increasing tile order, counts (host, ntiles entries) the
 * nonzeros of each tile. */
int sb_tile_partition(uint32_t nmodes, uint64_t nnz, uint32_t * const * inds,
    void const * vals, int vt, uint64_t const * tsize, uint32_t const * tdim,
    uint64_t ntiles, uint32_t * const * inds_out, void * vals_out, uint64_t * counts)
{
  if(nmodes < 1 || nmodes > SB_MAX_NMODES || nnz == 0 || nnz >= 0xffffffffull ||
      ntiles == 0 || ntiles > (1ull << 24)) {
    return SB_EINPUT;
  }
  TileGeom g;
  memset(&g, 0, sizeof(g));
  g.nmodes = nmodes;
  uint64_t prod = 1;
  for(uint32_t m = 0; m < nmodes; ++m) {
    if(tdim[m] == 0 || tsize[m] == 0) { return SB_EINPUT; }
    g.inds[m] = inds[m];
    g.tsize[m] = tsize[m];
    g.tdim[m] = tdim[m];
    prod *= tdim[m];
  }
  if(prod != ntiles) { return SB_EINPUT; }
  cudaStream_t s = stream();
  unsigned const nb = blocks_for(nnz, 256);
  uint32_t * id = nullptr, * perm = nullptr, * id2 = nullptr, * perm2 = nullptr;
  uint32_t * dcount = nullptr;
  int rc = SB_OK;
#define SB_STEP(x) do { rc = (x); if(rc) { goto done; } } while(0)
  SB_STEP(talloc(&id, nnz));
  SB_STEP(talloc(&perm, nnz));
  SB_STEP(talloc(&id2, nnz));
  SB_STEP(talloc(&perm2, nnz));
  SB_STEP(talloc(&dcount, ntiles));
  SB_TRY(cudaMemsetAsync(dcount, 0, ntiles * sizeof(uint32_t), s));
  k_tile_id<<<nb, 256, 0, s>>>(g, nnz, id, dcount);
  k_iota<<<nb, 256, 0, s>>>(perm, nnz);
  {
    int alt = 0;
    int const bits = ceil_log2(ntiles);
    if(bits > 0) {
      SB_STEP(sb_radix_sort_pairs(id, perm, id2, perm2, nnz, bits, &alt));
      if(alt) { uint32_t * t = perm; perm = perm2; perm2 = t; }
    }
  }
  for(uint32_t m = 0; m < nmodes; ++m) {
    k_gather_u32<<<nb, 256, 0, s>>>(inds[m], perm, inds_out[m], nnz);
  }
  if(vt == SB_F64) {
    k_gather_val<double><<<nb, 256, 0, s>>>((double const *) vals, perm, (double *) vals_out, nnz);
  } else {
    k_gather_val<float><<<nb, 256, 0, s>>>((float const *) vals, perm, (float *) vals_out, nnz);
  }
  SB_CHECK_LAUNCH();
  {
    uint32_t * h = (uint32_t *) malloc(ntiles * sizeof(uint32_t));
    if(!h) { rc = SB_ENOMEM; goto done; }
    cudaError_t const e1 = cudaMemcpyAsync(h, dcount, ntiles * sizeof(uint32_t),
                                           cudaMemcpyDeviceToHost, s);
    cudaError_t const e2 = e1 == cudaSuccess ? cudaStreamSynchronize(s) : e1;
    if(e2 != cudaSuccess) { free(h); rc = fail(e2); goto done; }
    for(uint64_t t = 0; t < ntiles; ++t) { counts[t] = h[t]; }
    free(h);
  }
done:
#undef SB_STEP
  tfree(id); tfree(perm); tfree(id2); tfree(perm2); tfree(dcount);
  return rc;
}

} /* extern "C" */
