/*
 * splatt_cli.c -- the `splatt` command line of the AdaTM build, on the B200
 * library (libadatm_b200.so) through its C ABI:
 *
 *   splatt cpd TENSOR [-i NITERS] [--tol TOL] [-r RANK] [-t NTHREADS] [-v] [--nowrite]
 *   splatt bench TENSOR -a adatm [-i NITERS] [-r RANK] [-t NTHREADS]
 *
 * `cpd` follows the reference's splatt_cpd_cmd_adaptive
 * (src/cmds/cmd_cpd.c:123-261): read the tensor, decide_product_order,
 * decide_parameters_auto (strategy 1), csf_alloc_adaptive,
 * rcsf_alloc_adaptive, decide_use_csfs, splatt_cpd_als_adaptive, then write
 * lambda.mat and mode<N>.mat unless --nowrite. `bench` follows splatt_bench
 * (src/cmds/cmd_bench.c:202-289) for the adatm algorithm: random factors of
 * the given rank, then bench_adaptm. Options and defaults are the
 * reference's (cmd_cpd.c:23-31, cmd_bench.c:75-87,212-215); the thread count
 * is accepted and ignored by GPU work, tiling and reordering are refused.
 *
 * Tensors are FROSTT-style text: one nonzero per line, N 1-based indices then
 * the value; '#' starts a comment line. Matrices are written as text, one row
 * per line, values "%0.8e" separated by spaces (SPLATT's own writer is not in
 * the reference, so its exact formatting is not reproduced).
 */
#define _GNU_SOURCE
#include <getopt.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "adatm_b200.h"

#define DEFAULT_ITERS 50
#define DEFAULT_TOL 1e-5
#define DEFAULT_RANK 10
#define BENCH_ITERS 5
#define BENCH_RANK 16

static void print_header(void) {
  printf("****************************************************************\n");
  printf("splatt (AdaTM on B200)\n\n");
}

/* Read a .tns file into a sptensor_t (dims = largest index per mode). */
static sptensor_t *read_tns(const char *fname) {
  FILE *f = fopen(fname, "r");
  if (!f) {
    fprintf(stderr, "SPLATT ERROR: unable to open '%s'\n", fname);
    return NULL;
  }
  char *line = NULL;
  size_t cap = 0;
  idx_t nmodes = 0, nnz = 0, alloc = 0;
  idx_t *ind[SPLATT_MAX_NMODES] = {0};
  val_t *vals = NULL;
  while (getline(&line, &cap, f) > 0) {
    char *p = line;
    while (*p == ' ' || *p == '\t') ++p;
    if (*p == '#' || *p == '\n' || *p == '\0') continue;
    double tok[SPLATT_MAX_NMODES + 1];
    idx_t nt = 0;
    while (nt < SPLATT_MAX_NMODES + 1) {
      char *end;
      const double v = strtod(p, &end);
      if (end == p) break;
      tok[nt++] = v;
      p = end;
    }
    if (nt < 2) continue;
    if (nmodes == 0) nmodes = nt - 1;
    if (nt != nmodes + 1) {
      fprintf(stderr, "SPLATT ERROR: '%s' line %lu has %lu fields, expected %lu\n", fname,
              (unsigned long)(nnz + 1), (unsigned long)nt, (unsigned long)(nmodes + 1));
      goto fail;
    }
    if (nnz == alloc) {
      alloc = alloc ? 2 * alloc : 1024;
      for (idx_t m = 0; m < nmodes; ++m) ind[m] = realloc(ind[m], alloc * sizeof(idx_t));
      vals = realloc(vals, alloc * sizeof(val_t));
      for (idx_t m = 0; m < nmodes; ++m)
        if (!ind[m]) goto oom;
      if (!vals) goto oom;
    }
    for (idx_t m = 0; m < nmodes; ++m) {
      if (tok[m] < 1) {
        fprintf(stderr, "SPLATT ERROR: '%s' has an index below 1\n", fname);
        goto fail;
      }
      ind[m][nnz] = (idx_t)tok[m] - 1;
    }
    vals[nnz] = tok[nmodes];
    ++nnz;
  }
  free(line);
  fclose(f);
  if (nnz == 0) {
    fprintf(stderr, "SPLATT ERROR: '%s' holds no nonzeros\n", fname);
    return NULL;
  }
  sptensor_t *tt = calloc(1, sizeof(sptensor_t));
  tt->nnz = nnz;
  tt->nmodes = nmodes;
  tt->dims = calloc(nmodes, sizeof(idx_t));
  tt->ind = calloc(nmodes, sizeof(idx_t *));
  for (idx_t m = 0; m < nmodes; ++m) {
    tt->ind[m] = ind[m];
    for (idx_t n = 0; n < nnz; ++n)
      if (ind[m][n] + 1 > tt->dims[m]) tt->dims[m] = ind[m][n] + 1;
  }
  tt->vals = vals;
  tt->tiled = 0;
  tt->type = nmodes == 3 ? 0 : 1;
  return tt;
oom:
  fprintf(stderr, "SPLATT ERROR: out of memory reading '%s'\n", fname);
fail:
  free(line);
  fclose(f);
  for (idx_t m = 0; m < SPLATT_MAX_NMODES; ++m) free(ind[m]);
  free(vals);
  return NULL;
}

static void free_tns(sptensor_t *tt) {
  if (!tt) return;
  for (idx_t m = 0; m < tt->nmodes; ++m) free(tt->ind[m]);
  free(tt->ind);
  free(tt->dims);
  free(tt->vals);
  free(tt);
}

static int write_rows(const char *fname, const val_t *v, idx_t rows, idx_t cols) {
  FILE *f = fopen(fname, "w");
  if (!f) {
    fprintf(stderr, "SPLATT ERROR: unable to write '%s'\n", fname);
    return 0;
  }
  for (idx_t i = 0; i < rows; ++i) {
    for (idx_t j = 0; j < cols; ++j) fprintf(f, j ? " %0.8e" : "%0.8e", v[i * cols + j]);
    fputc('\n', f);
  }
  fclose(f);
  return 1;
}


/* ------------------------------------------------------------------------ */

enum { OPT_TOL = 254, OPT_NOWRITE = 253, OPT_TILE = 255 };

static int cmd_cpd(int argc, char **argv) {
  static const struct option lopts[] = {
      {"iters", required_argument, 0, 'i'},   {"tol", required_argument, 0, OPT_TOL},
      {"rank", required_argument, 0, 'r'},    {"threads", required_argument, 0, 't'},
      {"tile", no_argument, 0, OPT_TILE},     {"nowrite", no_argument, 0, OPT_NOWRITE},
      {"verbose", no_argument, 0, 'v'},       {"help", no_argument, 0, 'h'},
      {0, 0, 0, 0}};
  double *opts = splatt_default_opts();
  opts[SPLATT_OPTION_CSF_ALLOC] = SPLATT_ADAPTIVE_TIME_EFFICIENT;
  opts[SPLATT_OPTION_NITER] = DEFAULT_ITERS;
  opts[SPLATT_OPTION_TOLERANCE] = DEFAULT_TOL;
  idx_t nfactors = DEFAULT_RANK;
  int write = 1;
  int c;
  optind = 1;
  while ((c = getopt_long(argc, argv, "i:r:t:vh", lopts, NULL)) != -1) {
    const char *arg = (optarg && optarg[0] == '=') ? optarg + 1 : optarg;
    switch (c) {
      case 'i': opts[SPLATT_OPTION_NITER] = (double)atoi(arg); break;
      case OPT_TOL: opts[SPLATT_OPTION_TOLERANCE] = atof(arg); break;
      case 'r': nfactors = (idx_t)atoi(arg); break;
      case 't': opts[SPLATT_OPTION_NTHREADS] = (double)atoi(arg); break;
      case 'v': opts[SPLATT_OPTION_VERBOSITY] += 1; break;
      case OPT_NOWRITE: write = 0; break;
      case OPT_TILE:
        fprintf(stderr, "SPLATT: --tile is not supported by the AdaTM path (it requires NOTILE).\n");
        splatt_free_opts(opts);
        return 1;
      default:
        printf("Usage: splatt cpd TENSOR [-i NITERS] [--tol TOL] [-r RANK] [-t NTHREADS] [-v] "
               "[--nowrite]\n");
        splatt_free_opts(opts);
        return c == 'h' ? 0 : 1;
    }
  }
  if (optind != argc - 1) {
    fprintf(stderr, "Usage: splatt cpd TENSOR [options]\n");
    splatt_free_opts(opts);
    return 1;
  }
  printf("Use splatt_cpd_cmd_adaptive.\n");
  print_header();
  sptensor_t *tt = read_tns(argv[optind]);
  if (!tt) {
    splatt_free_opts(opts);
    return 1;
  }
  const idx_t nmodes = tt->nmodes;
  idx_t *po[SPLATT_MAX_NMODES];
  for (idx_t m = 0; m < nmodes; ++m) po[m] = malloc(2 * nmodes * sizeof(idx_t));
  decide_product_order(tt, po);
  group_properties *grp = NULL;
  const idx_t n_grp = decide_parameters_auto(tt, nfactors, 1, (idx_t const **)po, &grp);
  for (idx_t m = 0; m < nmodes; ++m) free(po[m]);
  if (n_grp == 0 || grp == NULL) {
    fprintf(stderr, "SPLATT: planning failed: %s\n", adatm_last_error());
    free_tns(tt);
    splatt_free_opts(opts);
    return 1;
  }
  printf("Optimal predicted grp_prop:\n");
  printf("n_grp: %lu\n", (unsigned long)n_grp);
  print_group_properties(grp, n_grp, nmodes, "Optimal grp_prop");
  idx_t n_csf = 0;
  splatt_csf *csf = csf_alloc_adaptive(tt, grp, n_grp, opts, &n_csf);
  if (csf == NULL) {
    fprintf(stderr, "SPLATT: csf_alloc_adaptive failed: %s\n", adatm_last_error());
    adatm_free_groups(grp, n_grp);
    free_tns(tt);
    splatt_free_opts(opts);
    return 1;
  }
  printf("n_csf: %lu\n", (unsigned long)n_csf);
  free_tns(tt);
  printf("** CSF **\n");
  printf("CSF-STORAGE: %zu bytes\n\n", csf_storage_adaptive(csf, n_csf, grp, (int)n_grp));
  stats_csf_adaptive(csf, n_csf);
  printf("\n");
  idx_t n_rcsf = 0;
  rcsf_seq_adaptive *rs = rcsf_alloc_adaptive(csf, nfactors, grp, n_grp, n_csf, opts, &n_rcsf);
  printf("n_rcsf: %lu\n", (unsigned long)n_rcsf);
  printf("** RCSF **\n");
  printf("RCSF-STORAGE: %zu bytes\n", rcsf_storage_adaptive(rs, n_rcsf));
  stats_rcsf_adaptive(rs, n_rcsf);
  printf("\n");
  fflush(stdout);
  idx_t use_csfs[SPLATT_MAX_NMODES], use_tags[SPLATT_MAX_NMODES];
  decide_use_csfs(nmodes, grp, (int)n_grp, n_csf, use_csfs, use_tags);
  iprint_array(use_csfs, nmodes, "use_csfs");
  iprint_array(use_tags, nmodes, "use_tags");
  splatt_kruskal k;
  const int ret = splatt_cpd_als_adaptive(csf, rs, n_csf, grp, n_grp, use_csfs, use_tags, nfactors,
                                          opts, &k);
  if (ret != SPLATT_SUCCESS) {
    fprintf(stderr, "splatt_cpd_als_adaptive returned %d (%s). Aborting.\n", ret,
            adatm_last_error());
    splatt_free_csf(csf, opts);
    adatm_free_groups(grp, n_grp);
    splatt_free_opts(opts);
    return 1;
  }
  printf("Final fit: %f\n", k.fit);
  int ok = 1;
  if (write) {
    ok &= write_rows("lambda.mat", k.lambda, nfactors, 1);
    for (idx_t m = 0; m < nmodes; ++m) {
      char name[64];
      snprintf(name, sizeof(name), "mode%lu.mat", (unsigned long)(m + 1));
      ok &= write_rows(name, k.factors[m], k.dims[m], nfactors);
    }
  }
  splatt_free_kruskal(&k);
  splatt_free_csf(csf, opts);
  adatm_free_groups(grp, n_grp);
  splatt_free_opts(opts);
  return ok ? 0 : 1;
}

static int cmd_bench(int argc, char **argv) {
  static const struct option lopts[] = {
      {"alg", required_argument, 0, 'a'},   {"iters", required_argument, 0, 'i'},
      {"mode", required_argument, 0, 'm'},  {"threads", required_argument, 0, 't'},
      {"rank", required_argument, 0, 'r'},  {"scale", no_argument, 0, 's'},
      {"tile", no_argument, 0, OPT_TILE},   {"write", no_argument, 0, 'w'},
      {"rtype", required_argument, 0, 'z'}, {"pfile", required_argument, 0, 'p'},
      {"help", no_argument, 0, 'h'},        {0, 0, 0, 0}};
  idx_t niters = BENCH_ITERS, rank = BENCH_RANK, nthreads = 1;
  int adatm = 0;
  int c;
  optind = 1;
  while ((c = getopt_long(argc, argv, "a:i:m:t:r:swz:p:h", lopts, NULL)) != -1) {
    switch (c) {
      case 'a':
        if (strcmp(optarg, "adatm") == 0) {
          adatm = 1;
        } else {
          fprintf(stderr, "SPLATT: algorithm '%s' is not recognized.\n"
                          "Run with '--help' for assistance.\n", optarg);
          return 1;
        }
        break;
      case 'i': niters = (idx_t)atoi(optarg); break;
      case 'r': rank = (idx_t)atoi(optarg); break;
      case 't': nthreads = (idx_t)atoi(optarg); break;
      case 'm': case 's': case 'w': break;
      case 'z': case 'p':
        fprintf(stderr, "SPLATT: reordering is not part of this build.\n");
        return 1;
      case OPT_TILE:
        fprintf(stderr, "SPLATT: --tile is not supported by the AdaTM path (it requires NOTILE).\n");
        return 1;
      default:
        printf("Usage: splatt bench TENSOR -a adatm [-i NITERS] [-r RANK] [-t NTHREADS]\n");
        return c == 'h' ? 0 : 1;
    }
  }
  if (optind != argc - 1) {
    fprintf(stderr, "Usage: splatt bench TENSOR -a adatm [options]\n");
    return 1;
  }
  print_header();
  sptensor_t *tt = read_tns(argv[optind]);
  if (!tt) return 1;
  bench_opts bo;
  memset(&bo, 0, sizeof(bo));
  bo.niters = niters;
  bo.threads = &nthreads;
  bo.nruns = 1;
  matrix_t *mats[SPLATT_MAX_NMODES + 1] = {0};
  idx_t maxdim = 0;
  uint64_t state = 0x9E3779B97F4A7C15ull;
  for (idx_t m = 0; m < tt->nmodes; ++m) {
    mats[m] = calloc(1, sizeof(matrix_t));
    mats[m]->I = tt->dims[m];
    mats[m]->J = rank;
    mats[m]->rowmajor = 1;
    mats[m]->vals = malloc(tt->dims[m] * rank * sizeof(val_t));
    for (idx_t i = 0; i < tt->dims[m] * rank; ++i) {
      state = state * 6364136223846793005ull + 1442695040888963407ull;
      mats[m]->vals[i] = (double)(state >> 11) * (1.0 / 9007199254740992.0);
    }
    if (tt->dims[m] > maxdim) maxdim = tt->dims[m];
  }
  mats[SPLATT_MAX_NMODES] = calloc(1, sizeof(matrix_t));
  mats[SPLATT_MAX_NMODES]->I = maxdim;
  mats[SPLATT_MAX_NMODES]->J = rank;
  mats[SPLATT_MAX_NMODES]->rowmajor = 1;
  mats[SPLATT_MAX_NMODES]->vals = calloc(maxdim * rank, sizeof(val_t));
  printf("Benchmarking ---------------------------------------------------\n");
  printf("RANK=%lu ITS=%lu\n", (unsigned long)rank, (unsigned long)niters);
  if (adatm) bench_adaptm(tt, mats, &bo);
  printf("\n");
  for (idx_t m = 0; m < tt->nmodes; ++m) {
    free(mats[m]->vals);
    free(mats[m]);
  }
  free(mats[SPLATT_MAX_NMODES]->vals);
  free(mats[SPLATT_MAX_NMODES]);
  free_tns(tt);
  return 0;
}

int main(int argc, char **argv) {
  if (argc < 2 || strcmp(argv[1], "help") == 0 || strcmp(argv[1], "--help") == 0) {
    printf("splatt -- AdaTM sparse tensor CPD on B200\n\n"
           "The available commands are:\n"
           "  cpd\t\tCompute the Canonical Polyadic Decomposition.\n"
           "  bench\t\tBenchmark MTTKRP algorithms (-a adatm).\n"
           "  help\t\tPrint this help message.\n");
    return argc < 2 ? 1 : 0;
  }
  if (strcmp(argv[1], "cpd") == 0) return cmd_cpd(argc - 1, argv + 1);
  if (strcmp(argv[1], "bench") == 0) return cmd_bench(argc - 1, argv + 1);
  fprintf(stderr, "SPLATT: unknown command '%s'.\n", argv[1]);
  return 1;
}
