/*
 * splatt_cmd.c -- the `splatt cpd` command of this library: the reference's
 * command-line front end for CPD (src/cmds/cmd_cpd.c:220-560), the flags it
 * takes and the calls it makes, over libsplatt_b200.
 *
 *   splatt cpd TENSOR [-r RANK] [-i ITERS] [--tol TOL] [--seed SEED]
 *                     [-t THREADS] [--csf one|two|all] [--tile] [-s STEM]
 *                     [--nowrite] [-v] [--inner-its N] [--inner-tol TOL]
 *                     [-b ROWS] [--con CON[,MODELIST]] [--reg REG,MULT[,MODELIST]]
 *                     [--stream MODE] [-f FORGET]
 *
 * With --stream=MODE (1-based) it runs splatt_cpd_stream, which writes
 * mode%d.mat itself (cmd_cpd.c:497-507); otherwise it loads the tensor into
 * CSF (splatt_csf_load), runs splatt_cpd and writes lambda.mat and
 * mode%d.mat (STEM.lambda.mat, STEM.mode%d.mat with -s), with the reference's
 * number formats (src/io.c:713-775).
 *
 * Constraint and regularization names follow the reference's tables
 * (src/cmds/cmd_cpd_constraint.h:131-147): nonneg (alias ntf), rowsimp,
 * colsimp; frob, l1 (alias lasso), ntf-frob, ntf-l1, smooth.  A MODELIST is
 * a comma-separated list of 1-based modes, all modes when empty
 * (cmd_cpd.c:36-70).  Which of them a solver accepts is the library's
 * business: it returns SPLATT_ERROR_BADINPUT for the rest.
 */
#include <getopt.h>
#include <stdbool.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../../include/splatt_b200.h"

#define CMD_MAX_ARGS 32

static void usage(FILE * f)
{
  fprintf(f,
      "usage: splatt cpd TENSOR [options]\n"
      "  -r, --rank=RANK          rank of the factorization (default 10)\n"
      "  -i, --iters=ITERS        maximum outer iterations (default 50)\n"
      "      --tol=TOL            convergence tolerance (default 1e-5)\n"
      "      --seed=SEED          random seed (default: time)\n"
      "  -t, --threads=N          accepted for compatibility (the device does the work)\n"
      "      --csf=one|two|all    CSF allocation (default two)\n"
      "      --tile               dense-tiled CSF\n"
      "  -s, --stem=PATH          prefix of the output files\n"
      "      --nowrite            write no output files\n"
      "  -v, --verbose            more output\n"
      "      --inner-its=N        maximum ADMM iterations\n"
      "      --inner-tol=TOL      ADMM tolerance\n"
      "  -b, --block=ROWS         rows per ADMM chunk (row-separable constraints)\n"
      "      --con=CON[,MODES]    nonneg | ntf | rowsimp | colsimp\n"
      "      --reg=REG,MULT[,MODES]  frob | l1 | lasso | ntf-frob | ntf-l1 | smooth\n"
      "      --stream=MODE        stream mode MODE (1-based) of the tensor\n"
      "  -f, --forget=WEIGHT      forgetting factor of the streamed mode (default 0.95)\n");
}

/* split "a,b,c" in place; returns the number of fields */
static int split_commas(char * s, char ** out, int max)
{
  int n = 0;
  for(char * tok = strtok(s, ","); tok && n < max; tok = strtok(NULL, ",")) { out[n++] = tok; }
  return n;
}

/* 1-based MODELIST -> 0-based modes; all modes when the list is empty */
static int parse_modes(char ** args, int n, splatt_idx_t * modes)
{
  if(n == 0) {
    for(int m = 0; m < 8; ++m) { modes[m] = (splatt_idx_t) m; }
    return 8;
  }
  for(int i = 0; i < n; ++i) {
    long long const v = strtoll(args[i], NULL, 10);
    if(v < 1 || v > 8) { return -1; }
    modes[i] = (splatt_idx_t) (v - 1);
  }
  return n;
}

static int add_constraint(char * arg, splatt_cpd_opts * o)
{
  char * f[CMD_MAX_ARGS];
  int const n = split_commas(arg, f, CMD_MAX_ARGS);
  if(n < 1) { return 0; }
  splatt_idx_t modes[CMD_MAX_ARGS];
  int const nm = parse_modes(f + 1, n - 1, modes);
  if(nm < 0) { fprintf(stderr, "SPLATT: bad mode list in --con.\n"); return 0; }
  splatt_error_type rc;
  if(strcmp(f[0], "nonneg") == 0 || strcmp(f[0], "ntf") == 0) {
    rc = splatt_register_nonneg(o, modes, (splatt_idx_t) nm);
  } else if(strcmp(f[0], "rowsimp") == 0) {
    rc = splatt_register_rowsimp(o, modes, (splatt_idx_t) nm);
  } else if(strcmp(f[0], "colsimp") == 0) {
    rc = splatt_register_colsimp(o, modes, (splatt_idx_t) nm);
  } else {
    fprintf(stderr, "SPLATT: constraint '%s' not found.\n", f[0]);
    return 0;
  }
  return rc == SPLATT_SUCCESS;
}

static int add_regularization(char * arg, splatt_cpd_opts * o)
{
  char * f[CMD_MAX_ARGS];
  int const n = split_commas(arg, f, CMD_MAX_ARGS);
  if(n < 2) { fprintf(stderr, "SPLATT: regularizations require 'MULT' parameter.\n"); return 0; }
  splatt_val_t const mult = (splatt_val_t) strtod(f[1], NULL);
  splatt_idx_t modes[CMD_MAX_ARGS];
  int const nm = parse_modes(f + 2, n - 2, modes);
  if(nm < 0) { fprintf(stderr, "SPLATT: bad mode list in --reg.\n"); return 0; }
  splatt_idx_t const k = (splatt_idx_t) nm;
  splatt_error_type rc;
  if(strcmp(f[0], "frob") == 0) { rc = splatt_register_frob(o, mult, modes, k); }
  else if(strcmp(f[0], "l1") == 0 || strcmp(f[0], "lasso") == 0) {
    rc = splatt_register_lasso(o, mult, modes, k);
  } else if(strcmp(f[0], "ntf-frob") == 0) { rc = splatt_register_ntf_frob(o, mult, modes, k); }
  else if(strcmp(f[0], "ntf-l1") == 0) { rc = splatt_register_ntf_lasso(o, mult, modes, k); }
  else if(strcmp(f[0], "smooth") == 0) { rc = splatt_register_smooth(o, mult, modes, k); }
  else {
    fprintf(stderr, "SPLATT: regularization '%s' not found.\n", f[0]);
    return 0;
  }
  return rc == SPLATT_SUCCESS;
}

static int write_outputs(char const * stem, splatt_kruskal const * k)
{
  char name[1024];
  snprintf(name, sizeof(name), stem ? "%s.lambda.mat" : "lambda.mat", stem);
  FILE * f = fopen(name, "w");
  if(!f) { fprintf(stderr, "SPLATT ERROR: failed to open '%s'\n.", name); return 0; }
  for(splatt_idx_t r = 0; r < k->rank; ++r) { fprintf(f, "%le\n", (double) k->lambda[r]); }
  fclose(f);
  for(splatt_idx_t m = 0; m < k->nmodes; ++m) {
    if(stem) { snprintf(name, sizeof(name), "%s.mode%llu.mat", stem, (unsigned long long) m + 1); }
    else { snprintf(name, sizeof(name), "mode%llu.mat", (unsigned long long) m + 1); }
    f = fopen(name, "w");
    if(!f) { fprintf(stderr, "SPLATT ERROR: failed to open '%s'\n.", name); return 0; }
    for(splatt_idx_t i = 0; i < k->dims[m]; ++i) {
      for(splatt_idx_t r = 0; r < k->rank; ++r) {
        fprintf(f, "%+0.8le ", (double) k->factors[m][i * k->rank + r]);
      }
      fprintf(f, "\n");
    }
    fclose(f);
  }
  return 1;
}

enum { O_SEED = 256, O_NOWRITE, O_TILE, O_TOL, O_STREAM, O_CSF, O_CON, O_REG, O_IITS, O_ITOL };

static int cmd_cpd(int argc, char ** argv)
{
  static struct option const longs[] = {
    {"help", no_argument, 0, 'h'}, {"stream", required_argument, 0, O_STREAM},
    {"forget", required_argument, 0, 'f'}, {"rank", required_argument, 0, 'r'},
    {"stem", required_argument, 0, 's'}, {"nowrite", no_argument, 0, O_NOWRITE},
    {"iters", required_argument, 0, 'i'}, {"tol", required_argument, 0, O_TOL},
    {"seed", required_argument, 0, O_SEED}, {"verbose", no_argument, 0, 'v'},
    {"threads", required_argument, 0, 't'}, {"csf", required_argument, 0, O_CSF},
    {"tile", no_argument, 0, O_TILE}, {"con", required_argument, 0, O_CON},
    {"reg", required_argument, 0, O_REG}, {"inner-its", required_argument, 0, O_IITS},
    {"inner-tol", required_argument, 0, O_ITOL}, {"block", required_argument, 0, 'b'},
    {0, 0, 0, 0}};
  double * opts = splatt_default_opts();
  splatt_global_opts * gopts = splatt_alloc_global_opts();
  splatt_cpd_opts * copts = splatt_alloc_cpd_opts();
  splatt_idx_t rank = 10, stream_mode = 8;
  double forget = 0.95;
  char const * stem = NULL;
  bool write = true, ok = true;
  int c;
  optind = 1;
  while(ok && (c = getopt_long(argc, argv, "hf:r:s:i:vt:b:", longs, NULL)) != -1) {
    char * arg = optarg;
    if(arg && arg[0] == '=') { ++arg; }          /* -i=50 works too, as in the reference */
    switch(c) {
    case 'h': usage(stdout); goto done;
    case 'i': copts->max_iterations = strtoull(arg, NULL, 10); break;
    case O_TOL: copts->tolerance = (splatt_val_t) atof(arg); break;
    case 't': gopts->num_threads = atoi(arg); opts[SPLATT_OPTION_NTHREADS] = atoi(arg); break;
    case 'v': if(gopts->verbosity < SPLATT_VERBOSITY_MAX) { gopts->verbosity += 1; } break;
    case O_TILE: opts[SPLATT_OPTION_TILE] = SPLATT_DENSETILE; break;
    case O_NOWRITE: write = false; break;
    case 's': stem = arg; break;
    case 'r': rank = strtoull(arg, NULL, 10); break;
    case O_CSF:
      if(strcmp(arg, "one") == 0) { opts[SPLATT_OPTION_CSF_ALLOC] = SPLATT_CSF_ONEMODE; }
      else if(strcmp(arg, "two") == 0) { opts[SPLATT_OPTION_CSF_ALLOC] = SPLATT_CSF_TWOMODE; }
      else if(strcmp(arg, "all") == 0) { opts[SPLATT_OPTION_CSF_ALLOC] = SPLATT_CSF_ALLMODE; }
      else { fprintf(stderr, "SPLATT: --csf option '%s' not recognized.\n", arg); ok = false; }
      break;
    case O_SEED: gopts->random_seed = atoi(arg); srand((unsigned) gopts->random_seed); break;
    case O_STREAM: stream_mode = strtoull(arg, NULL, 10) - 1; break;
    case 'f': forget = atof(arg); break;
    case O_IITS: copts->max_inner_iterations = strtoull(arg, NULL, 10); break;
    case O_ITOL: copts->inner_tolerance = (splatt_val_t) atof(arg); break;
    case 'b':
      for(int m = 0; m < 8; ++m) { copts->chunk_sizes[m] = strtoull(arg, NULL, 10); }
      break;
    case O_CON: ok = add_constraint(arg, copts); break;
    case O_REG: ok = add_regularization(arg, copts); break;
    default: ok = false; break;
    }
  }
  if(!ok || optind != argc - 1) {
    usage(stderr);
    ok = false;
    goto done;
  }
  char const * fname = argv[optind];
  splatt_error_type rc;
  if(stream_mode != 8) {
    printf("SPLATT-B200 streaming CPD: %s, rank %llu, stream mode %llu, forget %g\n", fname,
        (unsigned long long) rank, (unsigned long long) stream_mode + 1, forget);
    rc = splatt_cpd_stream(fname, rank, stream_mode, forget, copts, gopts);
  } else {
    splatt_idx_t nmodes = 0;
    splatt_csf * csf = NULL;
    rc = splatt_csf_load(fname, &nmodes, &csf, opts);
    if(rc == SPLATT_SUCCESS) {
      printf("SPLATT-B200 CPD: %s, %llu modes, %llu nonzeros, rank %llu\n", fname,
          (unsigned long long) nmodes, (unsigned long long) csf->nnz, (unsigned long long) rank);
      splatt_kruskal * k = splatt_alloc_cpd(csf, rank);
      rc = k ? splatt_cpd(csf, rank, copts, gopts, k) : SPLATT_ERROR_NOMEMORY;
      if(rc == SPLATT_SUCCESS) {
        printf("final fit: %0.5f\n", k->fit);
        if(write && !write_outputs(stem, k)) { rc = SPLATT_ERROR_BADINPUT; }
      }
      splatt_free_cpd(k);
      splatt_free_csf(csf, opts);
    }
  }
  if(rc != SPLATT_SUCCESS) {
    fprintf(stderr, "SPLATT: cpd failed (error %d: %s)\n", (int) rc,
        rc == SPLATT_ERROR_BADINPUT ? "bad input" :
        rc == SPLATT_ERROR_NOMEMORY ? "out of memory" : "device error");
    ok = false;
  }
done:
  splatt_free_cpd_opts(copts);
  splatt_free_global_opts(gopts);
  splatt_free_opts(opts);
  return ok ? EXIT_SUCCESS : EXIT_FAILURE;
}

int main(int argc, char ** argv)
{
  if(argc < 2 || strcmp(argv[1], "-h") == 0 || strcmp(argv[1], "--help") == 0) {
    usage(argc < 2 ? stderr : stdout);
    return argc < 2 ? EXIT_FAILURE : EXIT_SUCCESS;
  }
  if(strcmp(argv[1], "cpd") == 0) { return cmd_cpd(argc - 1, argv + 1); }
  fprintf(stderr, "splatt: unknown command '%s' (this build has: cpd)\n", argv[1]);
  return EXIT_FAILURE;
}
