/*
 * kstream.h -- device state of one streaming CPD (plain C, shared by the host
 * code and k_stream.cu).  Every pointer is device memory.  Factor-like
 * matrices (Anew, Aold, D, M, aux, init) are row-major rows x R of the
 * stream's value type (double or float); Grams and all reductions are double.
 */
#ifndef SPLATT_B200_KSTREAM_H
#define SPLATT_B200_KSTREAM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int N;                       /* modes */
  int sm;                      /* streamed (time) mode */
  int nns;                     /* number of non-streamed modes */
  int ns[8];                   /* the non-streamed modes, in order */
  uint32_t R;                  /* rank */
  void * Anew[8];              /* current factors (non-streamed modes) */
  void * Aold[8];              /* factors at the end of the previous slice */
  void * D[8];                 /* ADMM duals */
  uint32_t rows[8];            /* rows of each factor for this slice */
  uint32_t rows0[8];           /* rows before this slice's growth (0: none kept) */
  void * M;                    /* MTTKRP buffer (max rows x R) */
  void * aux;                  /* ADMM auxiliary */
  void * init;                 /* ADMM primal at iteration start */
  double * G[8];               /* Grams (R x R full); G[sm] is the temporal Gram */
  double * old_gram;           /* temporal Gram before this slice's update */
  double * H;                  /* historical cross Grams, (nns-1) x R x R */
  double * Ginv;               /* (Gram + rho I)^{-1} of the current mode */
  double * s;                  /* the time row (R) */
  void * sT;                   /* the time row in the value type */
  double * Mt;                 /* time-mode MTTKRP (R) */
  uint32_t * inds[8];          /* slice COO (uint32), time mode unused */
  void * vals;                 /* slice values (value type) */
  uint32_t nnz;
  double * red;                /* FP64 accumulators and scalars (SB_RED_SIZE) */
  unsigned * bar;              /* grid barrier count + generation */
  int * status;                /* [0] barrier error, [1] bad pivot + 1,
                                  [2] outer iterations, [3] inner iterations */
  double * time_out;           /* where the slice's time row is stored */
  double reg, forget, outer_tol, inner_tol;
  int max_outer, max_inner;
  int first_slice;
  int prox[8];                 /* per non-streamed mode: SB_PROX_* */
  double prox_mult[8];         /* row-separable kinds: the multiplier */
  uint32_t chunk[8];           /* row-separable kinds: rows per ADMM chunk */
} StreamArgs;

/* proximal operator of a non-streamed mode's ADMM (the reference's streaming
 * driver: src/cpd/stream/StreamCPD.cc:325-337) */
#define SB_PROX_MAXCOLNORM 0         /* columns with 2-norm > 1 scaled to 1 */
#define SB_PROX_MAXCOLNORM_NONNEG 1  /* negatives zeroed, then the same scaling */
/* kinds SB_PROX_LASSO .. SB_PROX_NTF_FROB are row-separable: the ADMM runs in
 * independent chunks of chunk[m] rows (admm.c:352-395) */
#define SB_PROX_LASSO 2              /* soft threshold at prox_mult / rho */
#define SB_PROX_ROWSIMP 3            /* each row onto the probability simplex */
#define SB_PROX_NTF_LASSO 4          /* v > prox_mult/rho ? v - prox_mult/rho : 0 */
#define SB_PROX_NTF_FROB 5           /* max(v * rho / (prox_mult + rho), 0) */
/* not row-separable: each column onto the probability simplex, single-chunk
 * ADMM with a grid reduction per round of the column thresholds */
#define SB_PROX_COLSIMP 6
/* the row-separable kinds (chunked ADMM) */
#define SB_PROX_CHUNKED(k) ((k) >= SB_PROX_LASSO && (k) <= SB_PROX_NTF_FROB)

enum {
  PH_NORM_PARTIAL = 0,
  PH_NORM_APPLY,
  PH_GRAM,
  PH_TIME_MTTKRP,
  PH_TIME_SOLVE,
  PH_ZERO_MT,
  PH_MODE_MTTKRP,
  PH_ADMM_FIRST,
  PH_ADMM_SECOND,
  PH_ADMM_CHUNKED,
  PH_MODE_FINISH,
  PH_EPILOGUE,
  PH_COLSIMP_ROUND,
  PH_COLSIMP_APPLY
};

/* red[] layout the host reads (see k_stream.cu) */
#define SB_RED_SIZE 1352
#define SB_RD_NRM 272        /* 4 x 4, ring by the slice's ADMM counter */
#define SB_RD_DACC 288       /* 2 x 8 x 2 by outer-iteration parity */
#define SB_RD_CHUNK 832      /* 8: chunked ADMM, sum of iterations x rows per mode */
#define SB_RD_SIMP 840       /* 4 x 128: column simplex rounds, sums then counts */
#define SB_SIMP_RING 4       /* round r's accumulator: SB_RD_SIMP + (r % SB_SIMP_RING) * 128 */

size_t sb_stream_smem(uint32_t R);
int sb_stream_threads(void);
/* co-resident blocks for the fused launch */
int sb_stream_blocks(uint32_t R, int vt);
/* PLAIN executor: launch one phase */
int sb_stream_phase(StreamArgs const * a, int vt, int phase, int mq, int flag,
    uint32_t extra, int k, int nblocks);
/* FUSED executor: the whole slice update in one cooperative launch */
int sb_stream_fused(StreamArgs const * a, int vt, int nblocks);
/* SCHEDULED executor (many streams, several slices each, one launch).
 * The argument block (device, 256-aligned) is laid out as ints:
 *   [0] chains C  [1] heavy-group threshold (blocks)  [2] groups  [3] capacity K
 *   [4] error word  [5..7] unused
 *   base[K] len[K]          chain c = items base[c] .. base[c]+len[c]-1,
 *                           the slices of one stream in order
 *   next[K] busy[K]         per chain: next slice, claimed flag (zero)
 *   prio[K]                 per chain: work estimate (claim order)
 *   mbox[SB_SCHED_MAXG]     per group: the item it runs (written by it)
 *   gbar[2*SB_SCHED_MAXG]   per group: barrier count + generation (zero)
 *   gstart[SB_SCHED_MAXG+1] group g owns blocks [gstart[g], gstart[g+1])
 * then, at SB_SCHED_HDR_BYTES(K), StreamArgs items[K].  Groups with at
 * least [1] blocks claim the heaviest unclaimed chain, smaller groups the
 * lightest. */
#define SB_SCHED_MAXG 1024
#define SB_SCHED_HDR_BYTES(cap) \
  ((((size_t) (8 + 5 * (size_t) (cap) + 4 * SB_SCHED_MAXG + 1) * sizeof(int)) + 255) / 256 * 256)
int sb_stream_sched(int * dblock, int vt, int nblocks, uint32_t Rmax);
/* CUDA graph of (H2D of the pinned argument block) + scheduled launch, on
 * the library stream; returns SB_OK or an error if capture is unsupported */
int sb_graph_capture_sched(void ** graph_exec, void * dst, void const * src_pinned,
    size_t bytes, int vt, int nblocks, uint32_t Rmax);
int sb_graph_launch(void * graph_exec);
void sb_graph_destroy(void * graph_exec);
int sb_h2d_async(void * dst, void const * src, size_t bytes);
int sb_event_query_done(void * ev);
/* per-slice error^2 of the latest slice (see splatt_b200_stream_local_errsq) */
int sb_stream_local_err(StreamArgs const * a, int vt, int nblocks, double xnormsq,
    double * out);

#ifdef __cplusplus
}
#endif
#endif
