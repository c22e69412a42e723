/*
 * io.c -- coordinate tensor readers (host side ingest).
 *
 * Formats follow src/io.c: text .tns/.coo (whitespace separated, one nonzero
 * per line, '#' comments, 0- or 1-indexed per mode detected from the minimum
 * index, dims = max index (+1 when 0-indexed); src/io.c:62-110, 273-348) and
 * binary .bin (int32 magic 0 = COORD, uint64 idx width, uint64 val width,
 * then nmodes, dims[nmodes], nnz, the index arrays mode by mode and the
 * values, each at the header's width; src/io.c:118-196, 388-560).
 * tt_remove_empty semantics: src/sptensor.c:190-252.
 */
#define _GNU_SOURCE
#include "sb_host.h"

static int p_has_suffix(char const * s, char const * suf)
{
  size_t const a = strlen(s), b = strlen(suf);
  return a >= b && strcmp(s + a - b, suf) == 0;
}

static splatt_coord * p_read_text(FILE * fin)
{
  char * line = NULL;
  size_t len = 0;
  ssize_t rd;
  idx_t nmodes = 0;
  while((rd = getline(&line, &len, fin)) != -1) {
    if(rd > 1 && line[0] != '#') {
      char * save = NULL;
      for(char * p = strtok_r(line, " \t\n", &save); p; p = strtok_r(NULL, " \t\n", &save)) {
        ++nmodes;
      }
      break;
    }
  }
  if(nmodes < 2 || nmodes - 1 > SPLATT_MAX_NMODES) { free(line); return NULL; }
  --nmodes;
  idx_t dims[SPLATT_MAX_NMODES], offs[SPLATT_MAX_NMODES];
  for(idx_t m = 0; m < nmodes; ++m) { dims[m] = 0; offs[m] = 1; }
  idx_t nnz = 0;
  rewind(fin);
  while((rd = getline(&line, &len, fin)) != -1) {
    if(rd > 1 && line[0] != '#') {
      char * p = line;
      for(idx_t m = 0; m < nmodes; ++m) {
        idx_t x = (idx_t) strtoull(p, &p, 10);
        if(x > dims[m]) { dims[m] = x; }
        if(x < offs[m]) { offs[m] = x; }
      }
      strtod(p, &p);
      ++nnz;
    }
  }
  for(idx_t m = 0; m < nmodes; ++m) {
    if(offs[m] == 0) { ++dims[m]; }
  }
  splatt_coord * tt = splatt_alloc_coord(nmodes, nnz);
  if(!tt) { free(line); return NULL; }
  for(idx_t m = 0; m < nmodes; ++m) { tt->dims[m] = dims[m]; }
  rewind(fin);
  idx_t n = 0;
  while((rd = getline(&line, &len, fin)) != -1 && n < nnz) {
    if(rd > 1 && line[0] != '#') {
      char * p = line;
      for(idx_t m = 0; m < nmodes; ++m) {
        tt->ind[m][n] = (idx_t) strtoull(p, &p, 10) - offs[m];
      }
      tt->vals[n++] = (val_t) strtod(p, &p);
    }
  }
  free(line);
  return tt;
}

static int p_read_idx(FILE * f, uint64_t w, idx_t * out, idx_t count)
{
  for(idx_t i = 0; i < count; ++i) {
    if(w == 4) {
      uint32_t x;
      if(fread(&x, 4, 1, f) != 1) { return 0; }
      out[i] = (idx_t) x;
    } else {
      uint64_t x;
      if(fread(&x, 8, 1, f) != 1) { return 0; }
      out[i] = (idx_t) x;
    }
  }
  return 1;
}

static splatt_coord * p_read_bin(FILE * f)
{
  int32_t magic;
  uint64_t iw, vw;
  if(fread(&magic, 4, 1, f) != 1 || magic != 0) { return NULL; }
  if(fread(&iw, 8, 1, f) != 1 || fread(&vw, 8, 1, f) != 1) { return NULL; }
  if((iw != 4 && iw != 8) || (vw != 4 && vw != 8)) { return NULL; }
  idx_t nmodes, nnz, dims[SPLATT_MAX_NMODES];
  if(!p_read_idx(f, iw, &nmodes, 1) || nmodes > SPLATT_MAX_NMODES || nmodes < 1) { return NULL; }
  if(!p_read_idx(f, iw, dims, nmodes) || !p_read_idx(f, iw, &nnz, 1)) { return NULL; }
  /* the rest of the file must hold nnz indices per mode and nnz values: a
   * count that does not fit is refused before anything is allocated */
  long const here = ftell(f);
  if(here < 0 || fseek(f, 0, SEEK_END) != 0) { return NULL; }
  long const end = ftell(f);
  if(end < here || fseek(f, here, SEEK_SET) != 0) { return NULL; }
  if(nnz > (uint64_t) (end - here) / (nmodes * iw + vw)) { return NULL; }
  splatt_coord * tt = splatt_alloc_coord(nmodes, nnz);
  if(!tt) { return NULL; }
  for(idx_t m = 0; m < nmodes; ++m) {
    tt->dims[m] = dims[m];
    if(!p_read_idx(f, iw, tt->ind[m], nnz)) { splatt_free_coord(tt); return NULL; }
    /* every index inside its mode's dimension */
    for(idx_t n = 0; n < nnz; ++n) {
      if(tt->ind[m][n] >= dims[m]) { splatt_free_coord(tt); return NULL; }
    }
  }
  for(idx_t n = 0; n < nnz; ++n) {
    if(vw == 4) {
      float x;
      if(fread(&x, 4, 1, f) != 1) { splatt_free_coord(tt); return NULL; }
      tt->vals[n] = (val_t) x;
    } else {
      double x;
      if(fread(&x, 8, 1, f) != 1) { splatt_free_coord(tt); return NULL; }
      tt->vals[n] = (val_t) x;
    }
  }
  return tt;
}

splatt_coord * sb_read_tensor(char const * fname)
{
  FILE * f = fopen(fname, "rb");
  if(!f) { return NULL; }
  splatt_coord * tt = p_has_suffix(fname, ".bin") ? p_read_bin(f) : p_read_text(f);
  fclose(f);
  return tt;
}

/* ---- device ingest ---------------------------------------------------------
 * The file is read into host memory once; every per-element step (text
 * parsing, the binary format's width conversion and range checks) runs on
 * the device, which receives the raw bytes. */

/* number of fields of the first line the text reader takes (getline length
 * > 1, first character not '#'), minus the value: the mode count */
static idx_t p_text_modes(char const * b, size_t n)
{
  size_t i = 0;
  while(i < n) {
    size_t z = i;
    while(z < n && b[z] != '\n') { ++z; }
    size_t const len = z - i + (z < n ? 1 : 0);
    if(len > 1 && b[i] != '#') {
      idx_t f = 0;
      int in = 0;
      for(size_t k = i; k < z; ++k) {
        int const sp = b[k] == ' ' || b[k] == '\t' || b[k] == '\r' || b[k] == '\v' ||
            b[k] == '\f';
        if(!sp && !in) { ++f; }
        in = !sp;
      }
      return f > 0 ? f - 1 : 0;
    }
    i = z + 1;
  }
  return 0;
}

static int p_read_all(FILE * f, char ** buf, size_t * n)
{
  if(fseek(f, 0, SEEK_END) != 0) { return 0; }
  long const end = ftell(f);
  if(end <= 0 || fseek(f, 0, SEEK_SET) != 0) { return 0; }
  *buf = malloc((size_t) end);
  if(!*buf) { return 0; }
  *n = fread(*buf, 1, (size_t) end, f);
  return *n == (size_t) end;
}

int sb_file_modes(char const * fname, idx_t * nmodes)
{
  *nmodes = 0;
  FILE * f = fopen(fname, "rb");
  if(!f) { return SB_EINPUT; }
  if(p_has_suffix(fname, ".bin")) {
    int32_t magic;
    uint64_t iw, vw;
    idx_t N = 0;
    if(fread(&magic, 4, 1, f) == 1 && magic == 0 && fread(&iw, 8, 1, f) == 1 &&
        fread(&vw, 8, 1, f) == 1 && (iw == 4 || iw == 8) && p_read_idx(f, iw, &N, 1)) {
      *nmodes = N;
    }
  } else {
    char * line = NULL;
    size_t len = 0;
    ssize_t rd;
    while((rd = getline(&line, &len, f)) != -1) {
      if(rd > 1 && line[0] != '#') {
        *nmodes = p_text_modes(line, (size_t) rd);
        break;
      }
    }
    free(line);
  }
  fclose(f);
  return (*nmodes >= 1 && *nmodes <= SPLATT_MAX_NMODES) ? SB_OK : SB_EINPUT;
}

int sb_read_tensor_device(char const * fname, idx_t * nmodes, idx_t * nnz, idx_t * dims,
    uint32_t ** dinds, void ** dvals)
{
  *nmodes = 0;
  *nnz = 0;
  *dvals = NULL;
  for(idx_t m = 0; m < SPLATT_MAX_NMODES; ++m) { dinds[m] = NULL; }
  FILE * f = fopen(fname, "rb");
  if(!f) { return SB_EINPUT; }
  int rc = SB_OK;
  if(!p_has_suffix(fname, ".bin")) {
    char * buf = NULL;
    size_t n = 0;
    int const ok = p_read_all(f, &buf, &n);
    fclose(f);
    idx_t const N = ok ? p_text_modes(buf, n) : 0;
    if(N < 1 || N > SPLATT_MAX_NMODES) { free(buf); return SB_EINPUT; }
    rc = sb_ensure_init();
    if(rc) { free(buf); return rc; }
    uint64_t d64[SPLATT_MAX_NMODES], cnt = 0, nfb = 0;
    double * v64 = NULL;
    rc = sb_parse_text(buf, n, (uint32_t) N, dinds, &v64, &cnt, d64, &nfb);
    free(buf);
    if(rc) { return rc; }
    if(SB_VT == SB_F64) {
      *dvals = v64;
    } else {
      rc = sb_malloc(dvals, cnt * sizeof(val_t));
      if(rc == SB_OK) { rc = sb_convert_vals(v64, SB_F64, *dvals, SB_VT, cnt); }
      sb_free(v64);
    }
    *nmodes = N;
    *nnz = cnt;
    for(idx_t m = 0; m < N; ++m) { dims[m] = d64[m]; }
    return rc;
  }
  /* binary: header on the host, the arrays' raw bytes to the device */
  int32_t magic;
  uint64_t iw, vw;
  rc = SB_EINPUT;
  idx_t N = 0, cnt = 0;
  if(fread(&magic, 4, 1, f) == 1 && magic == 0 && fread(&iw, 8, 1, f) == 1 &&
      fread(&vw, 8, 1, f) == 1 && (iw == 4 || iw == 8) && (vw == 4 || vw == 8) &&
      p_read_idx(f, iw, &N, 1) && N >= 1 && N <= SPLATT_MAX_NMODES &&
      p_read_idx(f, iw, dims, N) && p_read_idx(f, iw, &cnt, 1)) {
    long const here = ftell(f);
    long end = -1;
    if(here >= 0 && fseek(f, 0, SEEK_END) == 0) { end = ftell(f); }
    if(end >= here && fseek(f, here, SEEK_SET) == 0 &&
        cnt <= (uint64_t) (end - here) / (N * iw + vw) && cnt < 0xffffffffull) {
      rc = SB_OK;
    }
  }
  if(rc == SB_OK) { rc = sb_ensure_init(); }
  size_t const bytes = (size_t) cnt * (iw > vw ? iw : vw);
  void * host = rc == SB_OK ? malloc(bytes ? bytes : 1) : NULL;
  void * raw = NULL;
  if(rc == SB_OK && !host) { rc = SB_ENOMEM; }
  if(rc == SB_OK) { rc = sb_malloc(&raw, bytes ? bytes : 1); }
  for(idx_t m = 0; m < N && rc == SB_OK; ++m) {
    if(dims[m] >= 0xffffffffull) { rc = SB_EINPUT; break; }
    rc = fread(host, iw, cnt, f) == cnt ? SB_OK : SB_EINPUT;
    if(rc == SB_OK) { rc = sb_malloc((void **) &dinds[m], (cnt ? cnt : 1) * sizeof(uint32_t)); }
    if(rc == SB_OK && iw == 8) {
      rc = sb_h2d(raw, host, cnt * 8);
      if(rc == SB_OK) { rc = sb_narrow_u64(raw, dinds[m], cnt, dims[m]); }
    } else if(rc == SB_OK) {
      rc = sb_h2d(dinds[m], host, cnt * 4);
      if(rc == SB_OK) { rc = sb_check_u32(dinds[m], cnt, dims[m]); }
    }
  }
  if(rc == SB_OK) { rc = fread(host, vw, cnt, f) == cnt ? SB_OK : SB_EINPUT; }
  if(rc == SB_OK) { rc = sb_malloc(dvals, (cnt ? cnt : 1) * sizeof(val_t)); }
  if(rc == SB_OK) { rc = sb_h2d(raw, host, cnt * vw); }
  if(rc == SB_OK) { rc = sb_convert_vals(raw, vw == 8 ? SB_F64 : SB_F32, *dvals, SB_VT, cnt); }
  fclose(f);
  free(host);
  sb_free(raw);
  if(rc) {
    for(idx_t m = 0; m < SPLATT_MAX_NMODES; ++m) { sb_free(dinds[m]); dinds[m] = NULL; }
    sb_free(*dvals);
    *dvals = NULL;
    return rc;
  }
  *nmodes = N;
  *nnz = cnt;
  return SB_OK;
}

idx_t sb_remove_empty(splatt_coord * tt)
{
  idx_t removed = 0;
  for(idx_t m = 0; m < tt->nmodes; ++m) {
    idx_t const d = tt->dims[m];
    idx_t * lab = calloc(d ? d : 1, sizeof(idx_t));
    if(!lab) { return (idx_t) -1; }
    for(idx_t n = 0; n < tt->nnz; ++n) { lab[tt->ind[m][n]] = 1; }
    idx_t used = 0;
    for(idx_t i = 0; i < d; ++i) { used += lab[i]; }
    if(used == d) { free(lab); continue; }
    removed += d - used;
    idx_t next = 0;
    tt->indmap[m] = malloc((used ? used : 1) * sizeof(idx_t));
    if(!tt->indmap[m]) { free(lab); return (idx_t) -1; }
    for(idx_t i = 0; i < d; ++i) {
      if(lab[i]) { tt->indmap[m][next] = i; lab[i] = next++; }
    }
    for(idx_t n = 0; n < tt->nnz; ++n) { tt->ind[m][n] = lab[tt->ind[m][n]]; }
    tt->dims[m] = used;
    free(lab);
  }
  return removed;
}
