/*
 * sb_stream.h -- the streaming handle shared by stream.c (single stream) and
 * serve.c (batches of streams, the serving loop).
 */
#ifndef SPLATT_B200_SB_STREAM_H
#define SPLATT_B200_SB_STREAM_H
#include "sb_host.h"
#include "../kernels/kstream.h"

struct splatt_b200_stream {
  idx_t N, sm, R;
  idx_t cap[SPLATT_MAX_NMODES];
  idx_t prevdim[SPLATT_MAX_NMODES];
  int vt;
  size_t vb;
  int exec;
  int nblocks;
  StreamArgs a;
  /* slice buffers */
  uint32_t * dind[SPLATT_MAX_NMODES];
  void * dval;
  idx_t slice_cap;
  uint32_t * h_ind[SPLATT_MAX_NMODES];   /* pinned-free host staging */
  void * h_val;
  /* device history of time rows */
  double * d_time;
  idx_t time_cap;
  idx_t t;
  idx_t last_outer;
  idx_t inner_total;
  idx_t inner_mode[SPLATT_MAX_NMODES];   /* ADMM iterations per non-streamed mode */
  int err;
  double xnorm_last;
  double * d_err;
  val_t * h_rand;
  idx_t h_rand_cap;
  /* per-stream generator for new rows (0: glibc rand(), as SPLATT) */
  int private_rng;
  unsigned rng_state;
  size_t bytes;               /* device bytes held by this stream */
};


/* grow_mats for the slice dims `sdims`; make room for the time row */
int sbs_grow(splatt_b200_stream * s, idx_t const * sdims);
int sbs_time_room(splatt_b200_stream * s);
/* point the stream's StreamArgs at a device slice (fused executors) */
void sbs_set_slice(splatt_b200_stream * s, uint32_t nnz, uint32_t * const * dinds,
    void * dvals);
/* after a slice was launched */
void sbs_advance(splatt_b200_stream * s);
/* read the device status words into the handle; SB_EDEVICE if it failed */
int sbs_read_status(splatt_b200_stream * s);

#endif
