/*
 * k_read.cu -- coordinate-tensor ingest on the device: parsing the text
 * format, narrowing the binary format, and dropping empty slices.
 *
 * Replaces the host loops of tt_read's text reader (src/io.c:62-110: one
 * nonzero per line, '#' comment lines, whitespace-separated indices then the
 * value, each mode 0- or 1-indexed as its smallest index says), the binary
 * reader's element conversion (src/io.c:162-196) and tt_remove_empty
 * (src/sptensor.c:190-252: kept indices renumbered in increasing order).
 *
 * Text.  The file's bytes are copied to the device once.  A byte starts a
 * data line when it follows a newline (or is the first byte), is neither '#'
 * nor '\n', and is not the file's last byte -- the lines the host reader
 * takes (getline length > 1, first character not '#').  A scan of those
 * marks numbers the lines; one thread then parses each line: the indices as
 * strtoull does (leading white space, decimal digits) and the value as
 * strtod does, exactly, whenever the decimal significand has at most 19
 * digits, fits 2^53 and the decimal exponent is within +-22: then the value
 * is one IEEE multiplication or division of two exactly representable
 * doubles, hence the correctly rounded result strtod returns (Clinger's fast
 * path).  Any other line (longer significands, hexadecimal or special
 * values, anything malformed) is flagged and re-read on the host with
 * strtoull / strtod from the host copy of the same bytes, so every value is
 * bit-identical to the host reader's.
 */
#include "common.cuh"

#include <stdlib.h>
#include <string.h>

namespace sb {
namespace {

__device__ __forceinline__ bool rd_space(char c)
{
  return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}

__global__ void k_rd_starts(char const * __restrict__ b, uint64_t n, uint32_t * __restrict__ f)
{
  uint64_t const i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n) { return; }
  bool const start = (i == 0) || b[i - 1] == '\n';
  char const c = b[i];
  f[i] = (start && c != '#' && c != '\n' && i + 1 < n) ? 1u : 0u;
}

__global__ void k_rd_positions(uint32_t const * __restrict__ f, uint32_t const * __restrict__ pos,
    uint64_t n, uint64_t * __restrict__ line_start)
{
  uint64_t const i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(i < n && f[i]) { line_start[pos[i]] = i; }
}

/* 10^k, k = 0..22: every one exactly representable in binary64 */
__device__ __forceinline__ double rd_pow10(int k)
{
  double p = 1.;
  for(int i = 0; i < k; ++i) { p *= 10.; }
  return p;
}

/* One line: nmodes indices then the value.  ok = false sends it to the host. */
__global__ void k_rd_parse(char const * __restrict__ b, uint64_t nbytes,
    uint64_t const * __restrict__ line_start, uint64_t nlines, uint32_t nmodes,
    uint64_t * __restrict__ const * inds, double * __restrict__ vals,
    uint8_t * __restrict__ fallback, unsigned long long * __restrict__ nfallback)
{
  uint64_t const l = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(l >= nlines) { return; }
  uint64_t p = line_start[l];
  bool ok = true;
  for(uint32_t m = 0; m < nmodes && ok; ++m) {
    while(p < nbytes && rd_space(b[p]) && b[p] != '\n') { ++p; }
    uint64_t x = 0;
    int nd = 0;
    while(p < nbytes && b[p] >= '0' && b[p] <= '9') {
      uint64_t const d = (uint64_t) (b[p] - '0');
      if(x > (0xffffffffffffffffull - d) / 10ull) { ok = false; break; }
      x = x * 10ull + d;
      ++nd;
      ++p;
    }
    if(nd == 0) { ok = false; }
    inds[m][l] = x;
  }
  double v = 0.;
  if(ok) {
    while(p < nbytes && rd_space(b[p]) && b[p] != '\n') { ++p; }
    bool neg = false;
    if(p < nbytes && (b[p] == '+' || b[p] == '-')) { neg = b[p] == '-'; ++p; }
    uint64_t w = 0;
    int sig = 0, frac = 0, ndig = 0;
    bool dot = false;
    while(p < nbytes) {
      char const c = b[p];
      if(c >= '0' && c <= '9') {
        ++ndig;
        if(sig > 0 || c != '0') {
          if(sig == 19) { ok = false; break; }
          w = w * 10ull + (uint64_t) (c - '0');
          ++sig;
        }
        if(dot) { ++frac; }
        ++p;
      } else if(c == '.' && !dot) {
        dot = true;
        ++p;
      } else {
        break;
      }
    }
    if(ndig == 0) { ok = false; }
    int e10 = 0;
    if(ok && p < nbytes && (b[p] == 'e' || b[p] == 'E')) {
      uint64_t q = p + 1;
      bool eneg = false;
      if(q < nbytes && (b[q] == '+' || b[q] == '-')) { eneg = b[q] == '-'; ++q; }
      int ed = 0, ev = 0;
      while(q < nbytes && b[q] >= '0' && b[q] <= '9') {
        if(ev < 100000) { ev = ev * 10 + (b[q] - '0'); }
        ++ed;
        ++q;
      }
      if(ed > 0) { e10 = eneg ? -ev : ev; p = q; }
    }
    /* the character after the number must end the field as strtod would
     * stop there: white space, end of line or end of file; anything else
     * (hexadecimal, inf, nan, stray text) goes to the host */
    if(ok && p < nbytes && !rd_space(b[p])) { ok = false; }
    if(ok) {
      int const q = e10 - frac;
      if(w == 0) {
        v = 0.;
      } else if(w <= (1ull << 53) && q >= -22 && q <= 22) {
        double const dw = (double) w;
        v = q >= 0 ? dw * rd_pow10(q) : dw / rd_pow10(-q);
      } else {
        ok = false;
      }
      if(neg) { v = -v; }
    }
  }
  vals[l] = v;
  fallback[l] = ok ? 0 : 1;
  if(!ok) { atomicAdd(nfallback, 1ull); }
}

__global__ void k_rd_minmax(uint64_t const * __restrict__ x, uint64_t n,
    unsigned long long * __restrict__ mn, unsigned long long * __restrict__ mx)
{
  unsigned long long lo = ~0ull, hi = 0ull;
  for(uint64_t i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += (uint64_t) gridDim.x * blockDim.x) {
    unsigned long long const v = x[i];
    lo = v < lo ? v : lo;
    hi = v > hi ? v : hi;
  }
  for(int o = 16; o > 0; o >>= 1) {
    unsigned long long const a = __shfl_xor_sync(0xffffffffu, lo, o);
    unsigned long long const c = __shfl_xor_sync(0xffffffffu, hi, o);
    lo = a < lo ? a : lo;
    hi = c > hi ? c : hi;
  }
  if((threadIdx.x & 31) == 0) { atomicMin(mn, lo); atomicMax(mx, hi); }
}

/* out = x - off as uint32 (the caller checked the range) */
__global__ void k_rd_shift(uint64_t const * __restrict__ x, uint64_t n, uint64_t off,
    uint32_t * __restrict__ out)
{
  uint64_t const i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(i < n) { out[i] = (uint32_t) (x[i] - off); }
}

__global__ void k_rd_mark(uint32_t const * __restrict__ ind, uint64_t n,
    uint32_t * __restrict__ used)
{
  uint64_t const i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(i < n) { used[ind[i]] = 1u; }
}

__global__ void k_rd_remap(uint32_t * __restrict__ ind, uint64_t n,
    uint32_t const * __restrict__ newid)
{
  uint64_t const i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(i < n) { ind[i] = newid[ind[i]]; }
}

__global__ void k_rd_indmap(uint32_t const * __restrict__ used, uint32_t const * __restrict__ newid,
    uint64_t d, uint32_t * __restrict__ indmap)
{
  uint64_t const i = (uint64_t) blockIdx.x * blockDim.x + threadIdx.x;
  if(i < d && used[i]) { indmap[newid[i]] = (uint32_t) i; }
}

} /* namespace */
} /* namespace sb */

using namespace sb;

extern "C" {

int sb_parse_text(char const * hbuf, uint64_t nbytes, uint32_t nmodes, uint32_t ** inds,
    double ** vals, uint64_t * nnz_out, uint64_t * dims, uint64_t * nfallback_out)
{
  *nnz_out = 0;
  for(uint32_t m = 0; m < nmodes; ++m) { inds[m] = nullptr; }
  *vals = nullptr;
  if(nmodes < 1 || nmodes > SB_MAX_NMODES || nbytes == 0 || nbytes >= 0xffffffffull) {
    return SB_EINPUT;
  }
  cudaStream_t const s = stream();
  char * db = nullptr;
  uint32_t * flag = nullptr, * pos = nullptr;
  uint64_t * start = nullptr;
  uint64_t * raw[SB_MAX_NMODES] = {nullptr};
  uint64_t ** draw = nullptr;
  uint8_t * fb = nullptr;
  unsigned long long * cnt = nullptr;
  uint64_t nl = 0;
  int rc = SB_OK;
#define RD(x) do { rc = (x); if(rc) { goto done; } } while(0)
  RD(talloc(&db, nbytes));
  RD(talloc(&flag, nbytes));
  RD(talloc(&pos, nbytes));
  SB_TRY(cudaMemcpyAsync(db, hbuf, nbytes, cudaMemcpyHostToDevice, s));
  k_rd_starts<<<blocks_for(nbytes, 256), 256, 0, s>>>(db, nbytes, flag);
  RD(sb_exclusive_scan_u32(flag, pos, nbytes, &nl));
  if(nl == 0 || nl >= 0xffffffffull) { rc = SB_EINPUT; goto done; }
  RD(talloc(&start, nl));
  k_rd_positions<<<blocks_for(nbytes, 256), 256, 0, s>>>(flag, pos, nbytes, start);
  tfree(flag); flag = nullptr;
  tfree(pos); pos = nullptr;
  for(uint32_t m = 0; m < nmodes; ++m) { RD(talloc(&raw[m], nl)); }
  RD(talloc(&draw, SB_MAX_NMODES));
  RD(talloc(vals, nl));
  RD(talloc(&fb, nl));
  RD(talloc(&cnt, 3));
  SB_TRY(cudaMemcpyAsync(draw, raw, sizeof(raw), cudaMemcpyHostToDevice, s));
  SB_TRY(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), s));
  k_rd_parse<<<blocks_for(nl, 128), 128, 0, s>>>(db, nbytes, start, nl, nmodes, draw, *vals, fb,
      cnt);
  SB_CHECK_LAUNCH();
  {
    unsigned long long nf = 0;
    SB_TRY(cudaMemcpyAsync(&nf, cnt, sizeof(nf), cudaMemcpyDeviceToHost, s));
    SB_TRY(cudaStreamSynchronize(s));
    *nfallback_out = nf;
    if(nf > 0) {
      /* the flagged lines, re-read on the host exactly as the host reader does */
      uint8_t * hf = (uint8_t *) malloc(nl);
      uint64_t * hs = (uint64_t *) malloc(nl * sizeof(uint64_t));
      if(!hf || !hs) { free(hf); free(hs); rc = SB_ENOMEM; goto done; }
      cudaError_t e = cudaMemcpyAsync(hf, fb, nl, cudaMemcpyDeviceToHost, s);
      if(e == cudaSuccess) { e = cudaMemcpyAsync(hs, start, nl * 8, cudaMemcpyDeviceToHost, s); }
      if(e == cudaSuccess) { e = cudaStreamSynchronize(s); }
      /* a private NUL-terminated copy of each flagged line for strtod */
      char * line = (char *) malloc(nbytes + 1);
      for(uint64_t l = 0; l < nl && e == cudaSuccess && line; ++l) {
        if(!hf[l]) { continue; }
        uint64_t a = hs[l], z = a;
        while(z < nbytes && hbuf[z] != '\n') { ++z; }
        memcpy(line, hbuf + a, z - a);
        line[z - a] = '\0';
        char * p = line;
        for(uint32_t m = 0; m < nmodes && e == cudaSuccess; ++m) {
          uint64_t const x = (uint64_t) strtoull(p, &p, 10);
          e = cudaMemcpyAsync(raw[m] + l, &x, 8, cudaMemcpyHostToDevice, s);
          if(e == cudaSuccess) { e = cudaStreamSynchronize(s); }
        }
        double const v = strtod(p, &p);
        if(e == cudaSuccess) { e = cudaMemcpyAsync(*vals + l, &v, 8, cudaMemcpyHostToDevice, s); }
        if(e == cudaSuccess) { e = cudaStreamSynchronize(s); }
      }
      free(line);
      free(hf);
      free(hs);
      if(e != cudaSuccess) { rc = fail(e); goto done; }
    }
  }
  /* dims and index base per mode: dims = largest index, +1 when some index
   * is 0 (the mode is 0-indexed), indices shifted down by 1 otherwise */
  for(uint32_t m = 0; m < nmodes; ++m) {
    unsigned long long mm[2] = {~0ull, 0ull};
    SB_TRY(cudaMemcpyAsync(cnt + 1, mm, sizeof(mm), cudaMemcpyHostToDevice, s));
    k_rd_minmax<<<148 * 4, 256, 0, s>>>(raw[m], nl, cnt + 1, cnt + 2);
    SB_TRY(cudaMemcpyAsync(mm, cnt + 1, sizeof(mm), cudaMemcpyDeviceToHost, s));
    SB_TRY(cudaStreamSynchronize(s));
    uint64_t const off = mm[0] == 0 ? 0 : 1;
    dims[m] = mm[1] + (off == 0 ? 1 : 0);
    if(dims[m] >= 0xffffffffull) { rc = SB_EINPUT; goto done; }
    RD(talloc(&inds[m], nl));
    k_rd_shift<<<blocks_for(nl, 256), 256, 0, s>>>(raw[m], nl, off, inds[m]);
    SB_CHECK_LAUNCH();
  }
  *nnz_out = nl;
done:
  tfree(db); tfree(flag); tfree(pos); tfree(start); tfree(draw); tfree(fb); tfree(cnt);
  for(uint32_t m = 0; m < nmodes; ++m) { tfree(raw[m]); }
  if(rc) {
    for(uint32_t m = 0; m < nmodes; ++m) { tfree(inds[m]); inds[m] = nullptr; }
    tfree(*vals);
    *vals = nullptr;
  }
#undef RD
  return rc;
}

int sb_remove_empty_device(uint32_t nmodes, uint64_t nnz, uint64_t * dims, uint32_t * const * inds,
    uint32_t ** indmap, uint64_t * removed)
{
  *removed = 0;
  cudaStream_t const s = stream();
  for(uint32_t m = 0; m < nmodes; ++m) {
    if(indmap) { indmap[m] = nullptr; }
    uint64_t const d = dims[m];
    if(d == 0 || nnz == 0) { continue; }
    uint32_t * used = nullptr, * nid = nullptr;
    int rc = talloc(&used, d);
    if(rc == SB_OK) { rc = talloc(&nid, d); }
    if(rc) { tfree(used); tfree(nid); return rc; }
    SB_TRY(cudaMemsetAsync(used, 0, d * sizeof(uint32_t), s));
    k_rd_mark<<<blocks_for(nnz, 256), 256, 0, s>>>(inds[m], nnz, used);
    uint64_t total = 0;
    rc = sb_exclusive_scan_u32(used, nid, d, &total);
    if(rc == SB_OK && total < d) {
      k_rd_remap<<<blocks_for(nnz, 256), 256, 0, s>>>(inds[m], nnz, nid);
      if(indmap) {
        rc = talloc(&indmap[m], total);
        if(rc == SB_OK) {
          k_rd_indmap<<<blocks_for(d, 256), 256, 0, s>>>(used, nid, d, indmap[m]);
        }
      }
      *removed += d - total;
      dims[m] = total;
    }
    tfree(used);
    tfree(nid);
    if(rc) { return rc; }
    SB_CHECK_LAUNCH();
  }
  return SB_OK;
}

} /* extern "C" */
