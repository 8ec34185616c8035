/*
 * splatt_shim.h -- the minimum of SPLATT v1.1.1's internal interface that the
 * reference's AdaTM files (adatm_rcsf.c, mttkrp.c, adatm_bench.c,
 * adatm_cpd.c, adatm_utils.c, adatm_sort.c, adatm_debug.c) need to compile.
 *
 * TEST INFRASTRUCTURE ONLY: it exists to build oracle/_ref, the reference's
 * own code used as a second checker of the oracle restatement. SPLATT itself
 * is not vendored with the reference; every type here is written from what
 * the AdaTM files read and write, and every function in ref_shim.c restates
 * the mathematics the AdaTM files expect of it.
 */
#ifndef ORACLE_SPLATT_SHIM_H
#define ORACLE_SPLATT_SHIM_H

#include <assert.h>
#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "splatt.h"

typedef splatt_idx_t idx_t;
typedef splatt_val_t val_t;
#define MAX_NMODES SPLATT_MAX_NMODES
#define SS_MIN(x, y) ((x) < (y) ? (x) : (y))
#define SS_MAX(x, y) ((x) > (y) ? (x) : (y))

void *splatt_malloc(size_t bytes);
void splatt_free(void *ptr);

/* timers */
typedef struct {
  int running;
  double seconds;
  double start;
  double stop;
} sp_timer_t;
typedef enum {
  TIMER_ALL, TIMER_CPD, TIMER_REORDER, TIMER_CONVERT, TIMER_MTTKRP,
  TIMER_INV, TIMER_FIT, TIMER_MATMUL, TIMER_ATA, TIMER_MATNORM, TIMER_IO,
  TIMER_PART, TIMER_MISC, TIMER_NTIMERS
} timer_id;
extern sp_timer_t timers[TIMER_NTIMERS];
void timer_reset(sp_timer_t *t);
void timer_start(sp_timer_t *t);
void timer_stop(sp_timer_t *t);
void timer_fstart(sp_timer_t *t);
void timer_inc_verbose(void);

/* tensors */
typedef enum { SPLATT_3MODE, SPLATT_NMODE } splatt_tt_type;
typedef struct {
  idx_t nnz;
  idx_t nmodes;
  idx_t *dims;
  idx_t **ind;
  val_t *vals;
  int tiled;
  splatt_tt_type type;
} sptensor_t;

typedef struct {
  idx_t nmodes;
  idx_t nnz;
  idx_t dims[MAX_NMODES];
  idx_t dim_perm[MAX_NMODES];
  idx_t *sptr;
  idx_t *fptr;
  idx_t *fids;
  idx_t *inds;
  val_t *vals;
  idx_t nslabs;
  idx_t *slabptr;
  idx_t *sids;
  int tiled;
} ftensor_t;

typedef struct {
  idx_t I;
  idx_t J;
  idx_t nnz;
  idx_t *rowptr;
  idx_t *colind;
  val_t *vals;
} spmatrix_t;

typedef struct {
  idx_t I;
  idx_t J;
  val_t *vals;
  int rowmajor;
} matrix_t;

typedef enum { MAT_NORM_2, MAT_NORM_MAX } splatt_mat_norm;

typedef struct {
  int rank;
} rank_info;

typedef struct {
  void **scratch;
  idx_t nscratch;
  sp_timer_t ttime;
} thd_info;

typedef enum { PERM_RAND, PERM_GRAPH, PERM_HGRAPH, PERM_FIBSCHED, PERM_ERROR } splatt_perm_type;
typedef struct {
  idx_t *perms[MAX_NMODES];
  idx_t *iperms[MAX_NMODES];
} permutation_t;

typedef struct {
  idx_t niters;
  idx_t *threads;
  idx_t nruns;
  int write;
  int tile;
  permutation_t *perm;
} bench_opts;

#define TILE_BEGIN ((idx_t)-2)
#define TILE_END ((idx_t)-1)
extern idx_t const TILE_SIZES[];
idx_t get_next_tileid(idx_t previd, idx_t const *tile_dims, idx_t nmodes,
                      idx_t iter_mode, idx_t mode_idx);

/* sorting / CSF */
void tt_sort(sptensor_t *tt, idx_t mode, idx_t *dim_perm);
idx_t csf_mode_depth(idx_t mode, idx_t const *perm, idx_t nmodes);
void csf_free(splatt_csf *csf, double const *opts);
val_t csf_frobsq(splatt_csf const *tensor);

/* dense matrices */
matrix_t *mat_alloc(idx_t nrows, idx_t ncols);
matrix_t *mat_rand(idx_t nrows, idx_t ncols);
void mat_free(matrix_t *mat);
void mat_aTa(matrix_t const *A, matrix_t *ret, rank_info *rinfo,
             thd_info *thds, idx_t nthreads);
void calc_gram_inv(idx_t mode, idx_t nmodes, matrix_t **aTa);
void mat_matmul(matrix_t const *A, matrix_t const *B, matrix_t *C);
void mat_normalize(matrix_t *A, val_t *lambda, splatt_mat_norm which,
                   rank_info *rinfo, thd_info *thds, idx_t nthreads);
void cpd_post_process(idx_t nfactors, idx_t nmodes, matrix_t **mats,
                      val_t *lambda, thd_info *thds, idx_t nthreads,
                      rank_info *rinfo);
matrix_t *perm_matrix(matrix_t const *mat, idx_t const *perm, matrix_t *retmat);
void mat_write(matrix_t const *mat, char const *fname);
void vec_write(val_t const *vec, idx_t len, char const *fname);

/* threads */
thd_info *thd_init(idx_t nthreads, idx_t nscratch, ...);
void thd_free(thd_info *thds, idx_t nthreads);
void thd_times(thd_info *thds, idx_t nthreads);
void thd_reset(thd_info *thds, idx_t nthreads);

/* util */
char *bytes_str(size_t bytes);
idx_t argmax_elem(idx_t const *arr, idx_t N);

#endif
