/*
 * ref_shim.c -- implementations behind shim/splatt_shim.h, so that the
 * reference's own AdaTM C files link into oracle/_ref/libadatm_ref.so.
 *
 * TEST INFRASTRUCTURE ONLY (the second checker of the oracle restatement).
 * SPLATT v1.1.1 is not vendored with the reference; each function below
 * restates the mathematics that the AdaTM files rely on (sorting, Gram
 * matrices, the Cholesky-based Gram inverse, column normalisation, the CSF
 * free and norm) in the same way the oracle does, and carries no SPLATT code.
 */
#include <omp.h>
#include <stdarg.h>
#include <stdint.h>
#include <time.h>

#include "adatm_oracle.h"
#include "splatt_shim.h"

sp_timer_t timers[TIMER_NTIMERS];
idx_t const TILE_SIZES[] = {1024, 1024, 1024};

void *splatt_malloc(size_t bytes) { return malloc(bytes ? bytes : 1); }
void splatt_free(void *ptr) { free(ptr); }

static double shim_now(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
void timer_reset(sp_timer_t *t) { memset(t, 0, sizeof(*t)); }
void timer_start(sp_timer_t *t) {
  if (!t->running) {
    t->running = 1;
    t->start = shim_now();
  }
}
void timer_stop(sp_timer_t *t) {
  if (t->running) {
    t->running = 0;
    t->stop = shim_now();
    t->seconds += t->stop - t->start;
  }
}
void timer_fstart(sp_timer_t *t) {
  timer_reset(t);
  timer_start(t);
}
void timer_inc_verbose(void) {}

idx_t get_next_tileid(idx_t previd, idx_t const *tile_dims, idx_t nmodes,
                      idx_t iter_mode, idx_t mode_idx) {
  (void)previd; (void)tile_dims; (void)nmodes; (void)iter_mode; (void)mode_idx;
  return TILE_END;
}

/* Lexicographic sort of the COO nonzeros by dim_perm (what the AdaTM files
 * expect of tt_sort at adatm_rcsf.c:179, adatm_bench.c:179,222). */
void tt_sort(sptensor_t *tt, idx_t mode, idx_t *dim_perm) {
  (void)mode;
  int const N = (int)tt->nmodes;
  uint64_t const nnz = tt->nnz;
  uint64_t *flat = (uint64_t *)malloc((size_t)N * nnz * sizeof(uint64_t) + 8);
  for (int m = 0; m < N; ++m) memcpy(flat + (uint64_t)m * nnz, tt->ind[m], nnz * sizeof(uint64_t));
  uint64_t *order = (uint64_t *)malloc(nnz * sizeof(uint64_t) + 8);
  orc_sort_order(N, nnz, tt->dims, flat, dim_perm, order);
  for (int m = 0; m < N; ++m)
    for (uint64_t i = 0; i < nnz; ++i) tt->ind[m][i] = flat[(uint64_t)m * nnz + order[i]];
  double *v = (double *)malloc(nnz * sizeof(double) + 8);
  for (uint64_t i = 0; i < nnz; ++i) v[i] = tt->vals[order[i]];
  memcpy(tt->vals, v, nnz * sizeof(double));
  free(v);
  free(order);
  free(flat);
}

idx_t csf_mode_depth(idx_t mode, idx_t const *perm, idx_t nmodes) {
  for (idx_t m = 0; m < nmodes; ++m)
    if (perm[m] == mode) return m;
  return MAX_NMODES;
}

void csf_free(splatt_csf *csf, double const *opts) {
  (void)csf;
  (void)opts; /* the driver frees the arrays it owns */
}

val_t csf_frobsq(splatt_csf const *tensor) {
  val_t s = 0;
  for (idx_t n = 0; n < tensor->nnz; ++n) s += tensor->pt->vals[n] * tensor->pt->vals[n];
  return s;
}

matrix_t *mat_alloc(idx_t nrows, idx_t ncols) {
  matrix_t *m = (matrix_t *)malloc(sizeof(matrix_t));
  m->I = nrows;
  m->J = ncols;
  m->rowmajor = 1;
  m->vals = (val_t *)calloc(nrows * ncols + 1, sizeof(val_t));
  return m;
}
matrix_t *mat_rand(idx_t nrows, idx_t ncols) {
  static uint64_t calls = 0;
  matrix_t *m = mat_alloc(nrows, ncols);
  orc_factor_init(0, calls++, nrows, ncols, m->vals);
  return m;
}
void mat_free(matrix_t *mat) {
  if (!mat) return;
  free(mat->vals);
  free(mat);
}

void mat_aTa(matrix_t const *A, matrix_t *ret, rank_info *rinfo, thd_info *thds,
             idx_t nthreads) {
  (void)rinfo; (void)thds; (void)nthreads;
  idx_t const R = A->J;
  memset(ret->vals, 0, R * R * sizeof(val_t));
  for (idx_t i = 0; i < A->I; ++i)
    for (idx_t a = 0; a < R; ++a)
      for (idx_t b = 0; b < R; ++b) ret->vals[a * R + b] += A->vals[i * R + a] * A->vals[i * R + b];
}

/* Hadamard product of every Gram matrix but `mode`, inverted through its
 * Cholesky factor, written to aTa[MAX_NMODES]. */
void calc_gram_inv(idx_t mode, idx_t nmodes, matrix_t **aTa) {
  idx_t const R = aTa[0]->J;
  double *V = (double *)calloc(R * R, sizeof(double));
  double *L = (double *)calloc(R * R, sizeof(double));
  double *y = (double *)calloc(R, sizeof(double));
  double *X = aTa[MAX_NMODES]->vals;
  for (idx_t x = 0; x < R * R; ++x) V[x] = 1.0;
  for (idx_t m = 0; m < nmodes; ++m) {
    if (m == mode) continue;
    for (idx_t x = 0; x < R * R; ++x) V[x] *= aTa[m]->vals[x];
  }
  for (idx_t j = 0; j < R; ++j) {
    double s = V[j * R + j];
    for (idx_t k = 0; k < j; ++k) s -= L[j * R + k] * L[j * R + k];
    L[j * R + j] = sqrt(s);
    for (idx_t i = j + 1; i < R; ++i) {
      double t = V[i * R + j];
      for (idx_t k = 0; k < j; ++k) t -= L[i * R + k] * L[j * R + k];
      L[i * R + j] = t / L[j * R + j];
    }
  }
  for (idx_t c = 0; c < R; ++c) {
    for (idx_t i = 0; i < R; ++i) {
      double t = (i == c) ? 1.0 : 0.0;
      for (idx_t k = 0; k < i; ++k) t -= L[i * R + k] * y[k];
      y[i] = t / L[i * R + i];
    }
    for (int64_t i = (int64_t)R - 1; i >= 0; --i) {
      double t = y[i];
      for (idx_t k = (idx_t)i + 1; k < R; ++k) t -= L[k * R + (idx_t)i] * X[k * R + c];
      X[(idx_t)i * R + c] = t / L[(idx_t)i * R + (idx_t)i];
    }
  }
  free(y);
  free(L);
  free(V);
}

void mat_matmul(matrix_t const *A, matrix_t const *B, matrix_t *C) {
  idx_t const I = A->I, K = A->J, J = B->J;
  C->I = I;
  for (idx_t i = 0; i < I; ++i)
    for (idx_t j = 0; j < J; ++j) {
      double t = 0;
      for (idx_t k = 0; k < K; ++k) t += A->vals[i * K + k] * B->vals[k * J + j];
      C->vals[i * J + j] = t;
    }
}

void mat_normalize(matrix_t *A, val_t *lambda, splatt_mat_norm which,
                   rank_info *rinfo, thd_info *thds, idx_t nthreads) {
  (void)rinfo; (void)thds; (void)nthreads;
  idx_t const I = A->I, R = A->J;
  for (idx_t r = 0; r < R; ++r) lambda[r] = 0;
  if (which == MAT_NORM_2) {
    for (idx_t i = 0; i < I; ++i)
      for (idx_t r = 0; r < R; ++r) lambda[r] += A->vals[i * R + r] * A->vals[i * R + r];
    for (idx_t r = 0; r < R; ++r) lambda[r] = sqrt(lambda[r]);
  } else {
    for (idx_t i = 0; i < I; ++i)
      for (idx_t r = 0; r < R; ++r) lambda[r] = SS_MAX(lambda[r], A->vals[i * R + r]);
    for (idx_t r = 0; r < R; ++r) lambda[r] = SS_MAX(lambda[r], 1.0);
  }
  for (idx_t i = 0; i < I; ++i)
    for (idx_t r = 0; r < R; ++r) A->vals[i * R + r] /= lambda[r];
}

void cpd_post_process(idx_t nfactors, idx_t nmodes, matrix_t **mats,
                      val_t *lambda, thd_info *thds, idx_t nthreads,
                      rank_info *rinfo) {
  val_t *tmp = (val_t *)calloc(nfactors, sizeof(val_t));
  for (idx_t m = 0; m < nmodes; ++m) {
    mat_normalize(mats[m], tmp, MAT_NORM_2, rinfo, thds, nthreads);
    for (idx_t r = 0; r < nfactors; ++r) lambda[r] *= tmp[r];
  }
  free(tmp);
}

matrix_t *perm_matrix(matrix_t const *mat, idx_t const *perm, matrix_t *retmat) {
  (void)perm;
  if (!retmat) retmat = mat_alloc(mat->I, mat->J);
  memcpy(retmat->vals, mat->vals, mat->I * mat->J * sizeof(val_t));
  return retmat;
}
void mat_write(matrix_t const *mat, char const *fname) { (void)mat; (void)fname; }
void vec_write(val_t const *vec, idx_t len, char const *fname) { (void)vec; (void)len; (void)fname; }

thd_info *thd_init(idx_t nthreads, idx_t nscratch, ...) {
  thd_info *thds = (thd_info *)calloc(nthreads, sizeof(thd_info));
  size_t sizes[16];
  va_list ap;
  va_start(ap, nscratch);
  for (idx_t s = 0; s < nscratch && s < 16; ++s) sizes[s] = va_arg(ap, size_t);
  va_end(ap);
  for (idx_t t = 0; t < nthreads; ++t) {
    thds[t].nscratch = nscratch;
    thds[t].scratch = (void **)calloc(nscratch, sizeof(void *));
    for (idx_t s = 0; s < nscratch; ++s) thds[t].scratch[s] = calloc(sizes[s] + 64, 1);
  }
  return thds;
}
void thd_free(thd_info *thds, idx_t nthreads) {
  for (idx_t t = 0; t < nthreads; ++t) {
    for (idx_t s = 0; s < thds[t].nscratch; ++s) free(thds[t].scratch[s]);
    free(thds[t].scratch);
  }
  free(thds);
}
void thd_times(thd_info *thds, idx_t nthreads) { (void)thds; (void)nthreads; }
void thd_reset(thd_info *thds, idx_t nthreads) {
  for (idx_t t = 0; t < nthreads; ++t) timer_reset(&thds[t].ttime);
}

char *bytes_str(size_t bytes) {
  char *s = (char *)malloc(64);
  snprintf(s, 64, "%zu B", bytes);
  return s;
}
idx_t argmax_elem(idx_t const *arr, idx_t N) {
  idx_t mkr = 0;
  for (idx_t i = 1; i < N; ++i)
    if (arr[i] > arr[mkr]) mkr = i;
  return mkr;
}

double *splatt_default_opts(void) {
  double *o = (double *)calloc(SPLATT_OPTION_NOPTIONS, sizeof(double));
  o[SPLATT_OPTION_NTHREADS] = 1;
  o[SPLATT_OPTION_TOLERANCE] = 1e-5;
  o[SPLATT_OPTION_NITER] = 50;
  o[SPLATT_OPTION_VERBOSITY] = SPLATT_VERBOSITY_NONE;
  o[SPLATT_OPTION_CSF_ALLOC] = SPLATT_ADAPTIVE_TIME_EFFICIENT;
  o[SPLATT_OPTION_TILE] = SPLATT_NOTILE;
  return o;
}
void splatt_free_opts(double *opts) { free(opts); }
