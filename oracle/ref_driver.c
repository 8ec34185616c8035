/*
 * ref_driver.c -- ctypes-facing driver around the reference's own AdaTM
 * files, linked as oracle/_ref/libadatm_ref.so.
 *
 * TEST INFRASTRUCTURE ONLY: tests use it to pin the oracle restatement to
 * the reference code (plan choice, CSF arrays, MTTKRP and CP-ALS values), and
 * bench.py's CPU baseline may time it. Two reference defects are worked
 * around from outside, without touching the reference files:
 *  - memo buffers accumulate across calls (mttkrp.c:922,848 with
 *    adatm_rcsf.c:273-274): the link wraps mttkrp_csf_adaptive so that, when
 *    ref_zero_memo is set, the memo values of a memo-root call are zeroed
 *    before the call;
 *  - the N-mode memo root races across OpenMP threads (mttkrp.c:910,840,875):
 *    parity runs pass nthreads = 1.
 */
#include <omp.h>
#include <stdint.h>

#include "splatt_shim.h"
#include "adatm_rcsf.h"
#include "adatm_bench.h"
#include "adatm_cpd.h"
#include "mttkrp.h"

static int ref_zero_memo = 1;

void __real_mttkrp_csf_adaptive(splatt_csf const *tensors,
                                rcsf_seq_adaptive const *rs_seq, idx_t n_csf,
                                matrix_t **mats, idx_t mode, thd_info *thds,
                                group_properties *grp_prop, int n_grp,
                                idx_t use_csf, idx_t use_tag,
                                double const *opts);

void __wrap_mttkrp_csf_adaptive(splatt_csf const *tensors,
                                rcsf_seq_adaptive const *rs_seq, idx_t n_csf,
                                matrix_t **mats, idx_t mode, thd_info *thds,
                                group_properties *grp_prop, int n_grp,
                                idx_t use_csf, idx_t use_tag,
                                double const *opts) {
  if (ref_zero_memo && use_tag == 0 && grp_prop[use_csf].n_imten != 0) {
    rcsf_seq_adaptive const *seq = rs_seq + use_csf;
    for (idx_t d = 0; d < seq->n_imten; ++d)
      memset(seq->rcsfs[d].pt->vals, 0, seq->rcsfs[d].nnz * sizeof(val_t));
  }
  __real_mttkrp_csf_adaptive(tensors, rs_seq, n_csf, mats, mode, thds,
                             grp_prop, n_grp, use_csf, use_tag, opts);
}

typedef struct ref_state {
  sptensor_t tt;
  idx_t R;
  int nthreads;
  group_properties *grp;
  idx_t n_grp;
  splatt_csf *cs;
  idx_t n_csf;
  rcsf_seq_adaptive *rs;
  idx_t n_rcsf;
  idx_t use_csfs[MAX_NMODES];
  idx_t use_tags[MAX_NMODES];
  double *opts;
  thd_info *thds;
  matrix_t *mats[MAX_NMODES + 1];
} ref_state;

static void ref_fill_tt(sptensor_t *tt, int N, uint64_t nnz,
                        const uint64_t *dims, const uint64_t *inds,
                        const double *vals) {
  tt->nnz = nnz;
  tt->nmodes = (idx_t)N;
  tt->type = N == 3 ? SPLATT_3MODE : SPLATT_NMODE;
  tt->tiled = 0;
  tt->dims = (idx_t *)malloc(N * sizeof(idx_t));
  tt->ind = (idx_t **)malloc(N * sizeof(idx_t *));
  for (int m = 0; m < N; ++m) {
    tt->dims[m] = dims[m];
    tt->ind[m] = (idx_t *)malloc(nnz * sizeof(idx_t) + 8);
    memcpy(tt->ind[m], inds + (uint64_t)m * nnz, nnz * sizeof(idx_t));
  }
  tt->vals = (val_t *)malloc(nnz * sizeof(val_t) + 8);
  memcpy(tt->vals, vals, nnz * sizeof(val_t));
}

static void ref_free_tt(sptensor_t *tt) {
  for (idx_t m = 0; m < tt->nmodes; ++m) free(tt->ind[m]);
  free(tt->ind);
  free(tt->dims);
  free(tt->vals);
}

/* decide_product_order + decide_parameters_auto (strategy 1, as the CLI and
 * bench use). Writes n_grp, then per group memo_mode, begin_imten, n_imten,
 * o_opt[N]. Returns n_grp, or 0 for N == 3, where the reference's candidate
 * count reads an uninitialised value (adatm_bench.c:303-326). */
uint64_t ref_plan(int N, uint64_t nnz, const uint64_t *dims,
                  const uint64_t *inds, const double *vals, uint64_t R,
                  uint64_t *out) {
  if (N <= 3) return 0;
  sptensor_t tt;
  ref_fill_tt(&tt, N, nnz, dims, inds, vals);
  idx_t **po = (idx_t **)malloc(N * sizeof(idx_t *));
  for (int i = 0; i < N; ++i) po[i] = (idx_t *)malloc(2 * N * sizeof(idx_t));
  decide_product_order(&tt, po);
  group_properties *grp = NULL;
  idx_t const n_grp = decide_parameters_auto(&tt, R, 1, (idx_t const **)po, &grp);
  out[0] = n_grp;
  for (idx_t g = 0; g < n_grp; ++g) {
    uint64_t *o = out + 1 + g * (3 + N);
    o[0] = grp[g].memo_mode;
    o[1] = grp[g].begin_imten;
    o[2] = grp[g].n_imten;
    for (int m = 0; m < N; ++m) o[3 + m] = grp[g].o_opt[m];
    free(grp[g].o_opt);
  }
  free(grp);
  for (int i = 0; i < N; ++i) free(po[i]);
  free(po);
  ref_free_tt(&tt);
  return n_grp;
}

/* csf_alloc_adaptive + rcsf_alloc_adaptive + decide_use_csfs for the given
 * plan (same packing as ref_plan's output), TIME_EFFICIENT, no tiling. */
ref_state *ref_build(int N, uint64_t nnz, const uint64_t *dims,
                     const uint64_t *inds, const double *vals, uint64_t R,
                     const uint64_t *plan, int nthreads) {
  ref_state *st = (ref_state *)calloc(1, sizeof(ref_state));
  ref_fill_tt(&st->tt, N, nnz, dims, inds, vals);
  st->R = R;
  st->nthreads = nthreads;
  st->opts = splatt_default_opts();
  st->opts[SPLATT_OPTION_NTHREADS] = nthreads;
  st->opts[SPLATT_OPTION_CSF_ALLOC] = SPLATT_ADAPTIVE_TIME_EFFICIENT;
  st->opts[SPLATT_OPTION_TILE] = SPLATT_NOTILE;
  st->n_grp = plan[0];
  st->grp = (group_properties *)calloc(st->n_grp, sizeof(group_properties));
  for (idx_t g = 0; g < st->n_grp; ++g) {
    const uint64_t *o = plan + 1 + g * (3 + N);
    st->grp[g].memo_mode = o[0];
    st->grp[g].begin_imten = o[1];
    st->grp[g].n_imten = o[2];
    st->grp[g].o_opt = (idx_t *)malloc(N * sizeof(idx_t));
    for (int m = 0; m < N; ++m) st->grp[g].o_opt[m] = o[3 + m];
  }
  st->cs = csf_alloc_adaptive(&st->tt, st->grp, st->n_grp, st->opts, &st->n_csf);
  st->rs = rcsf_alloc_adaptive(st->cs, R, st->grp, st->n_grp, st->n_csf, st->opts, &st->n_rcsf);
  decide_use_csfs((idx_t)N, st->grp, (int)st->n_grp, st->n_csf, st->use_csfs, st->use_tags);
  omp_set_num_threads(nthreads);
  st->thds = thd_init(nthreads, 3, (R * R * sizeof(val_t)) + 64, (size_t)0,
                      (N * R * sizeof(val_t)) + 64);
  idx_t maxdim = 0;
  for (int m = 0; m < N; ++m) maxdim = SS_MAX(maxdim, dims[m]);
  for (int m = 0; m < N; ++m) st->mats[m] = mat_alloc(dims[m], R);
  st->mats[MAX_NMODES] = mat_alloc(maxdim, R);
  return st;
}

uint64_t ref_n_csf(ref_state *st) { return st->n_csf; }

/* Replace the per-mode trees and tags that ref_mttkrp / ref_cpd pass to the
 * reference (a caller's own use_csfs / use_tags instead of decide_use_csfs's). */
void ref_set_use(ref_state *st, const uint64_t *use_csfs, const uint64_t *use_tags) {
  for (idx_t m = 0; m < st->tt.nmodes; ++m) {
    st->use_csfs[m] = use_csfs[m];
    st->use_tags[m] = use_tags[m];
  }
}

void ref_use(ref_state *st, uint64_t *use_csfs, uint64_t *use_tags) {
  for (idx_t m = 0; m < st->tt.nmodes; ++m) {
    use_csfs[m] = st->use_csfs[m];
    use_tags[m] = st->use_tags[m];
  }
}

/* nfibs, dim_perm of CSF g; arrays copied out by ref_csf_array. */
void ref_csf_shape(ref_state *st, int g, uint64_t *nfibs, uint64_t *dim_perm) {
  splatt_csf const *ct = st->cs + g;
  for (idx_t l = 0; l < ct->nmodes; ++l) {
    nfibs[l] = ct->pt->nfibs[l];
    dim_perm[l] = ct->dim_perm[l];
  }
}
/* which: 0 = fptr[l] (nfibs[l]+1 entries), 1 = fids[l] (nfibs[l] entries;
 * returns 0 when the reference keeps it NULL). */
int ref_csf_array(ref_state *st, int g, int l, int which, uint64_t *out) {
  splatt_csf const *ct = st->cs + g;
  idx_t const n = ct->pt->nfibs[l] + (which == 0 ? 1 : 0);
  idx_t const *src = which == 0 ? ct->pt->fptr[l] : ct->pt->fids[l];
  if (src == NULL) return 0;
  memcpy(out, src, n * sizeof(idx_t));
  return 1;
}
void ref_csf_vals(ref_state *st, int g, double *out) {
  memcpy(out, st->cs[g].pt->vals, st->cs[g].nnz * sizeof(double));
}
/* memo tree shape: nmodes and nnz of rcsfs[deg] of sequence j */
void ref_memo_shape(ref_state *st, int j, int deg, uint64_t *out) {
  splatt_csf const *r = st->rs[j].rcsfs + deg;
  out[0] = r->nmodes;
  out[1] = r->nnz;
  out[2] = st->rs[j].begin_imten;
  out[3] = st->rs[j].n_imten;
}
void ref_memo_vals(ref_state *st, int j, int deg, double *out) {
  splatt_csf const *r = st->rs[j].rcsfs + deg;
  memcpy(out, r->pt->vals, r->nnz * sizeof(double));
}

static void ref_load_mats(ref_state *st, double *const *mats) {
  for (idx_t m = 0; m < st->tt.nmodes; ++m)
    memcpy(st->mats[m]->vals, mats[m], st->tt.dims[m] * st->R * sizeof(double));
}

/* mttkrp_csf_adaptive for `mode` with the plan's csf/tag; out is
 * dims[mode] x R. */
void ref_mttkrp(ref_state *st, double *const *mats, uint64_t mode, double *out,
                int zero_memo) {
  ref_zero_memo = zero_memo;
  ref_load_mats(st, mats);
  st->mats[MAX_NMODES]->I = st->tt.dims[mode];
  mttkrp_csf_adaptive(st->cs, st->rs, st->n_csf, st->mats, mode, st->thds,
                      st->grp, (int)st->n_grp, st->use_csfs[mode],
                      st->use_tags[mode], st->opts);
  memcpy(out, st->mats[MAX_NMODES]->vals, st->tt.dims[mode] * st->R * sizeof(double));
  ref_zero_memo = 1;
}

/* One timed MTTKRP sequence over all modes (the inner loop of bench_adaptm,
 * adatm_bench.c:613-633) on the factors already loaded; returns seconds. */
double ref_mttkrp_sequence(ref_state *st, int zero_memo) {
  ref_zero_memo = zero_memo;
  double const t0 = omp_get_wtime();
  for (idx_t m = 0; m < st->tt.nmodes; ++m) {
    st->mats[MAX_NMODES]->I = st->tt.dims[m];
    mttkrp_csf_adaptive(st->cs, st->rs, st->n_csf, st->mats, m, st->thds,
                        st->grp, (int)st->n_grp, st->use_csfs[m],
                        st->use_tags[m], st->opts);
  }
  double const t1 = omp_get_wtime();
  ref_zero_memo = 1;
  return t1 - t0;
}

/* cpd_als_iterate_adaptive on the given initial factors (overwritten with the
 * result); lambda receives R values; returns the final fit. */
double ref_cpd(ref_state *st, double *const *mats, double *lambda,
               uint64_t niters, double tol, int zero_memo) {
  ref_zero_memo = zero_memo;
  ref_load_mats(st, mats);
  st->opts[SPLATT_OPTION_NITER] = (double)niters;
  st->opts[SPLATT_OPTION_TOLERANCE] = tol;
  st->opts[SPLATT_OPTION_VERBOSITY] = SPLATT_VERBOSITY_NONE;
  rank_info rinfo;
  rinfo.rank = 0;
  double const fit = cpd_als_iterate_adaptive(
      st->cs, st->rs, st->n_csf, st->grp, st->n_grp, st->use_csfs,
      st->use_tags, st->mats, lambda, st->R, &rinfo, st->opts);
  for (idx_t m = 0; m < st->tt.nmodes; ++m)
    memcpy(mats[m], st->mats[m]->vals, st->tt.dims[m] * st->R * sizeof(double));
  ref_zero_memo = 1;
  return fit;
}

void ref_free(ref_state *st) {
  if (!st) return;
  for (idx_t j = 0; j < st->n_rcsf; ++j) {
    for (idx_t d = 0; d < st->rs[j].n_imten; ++d) {
      free(st->rs[j].rcsfs[d].pt->vals);
      free(st->rs[j].rcsfs[d].pt);
    }
    free(st->rs[j].rcsfs);
  }
  free(st->rs);
  for (idx_t g = 0; g < st->n_csf; ++g) {
    csf_sparsity *pt = st->cs[g].pt;
    /* the reference allocates pt without zeroing it: only fptr[0..N-2]
     * and fids[1..N-1] are set (adatm_rcsf.c:185-207, fids[0] is NULL) */
    for (idx_t l = 0; l + 1 < st->cs[g].nmodes; ++l) free(pt->fptr[l]);
    for (idx_t l = 1; l < st->cs[g].nmodes; ++l) free(pt->fids[l]);
    free(pt->vals);
    free(pt);
  }
  free(st->cs);
  for (idx_t g = 0; g < st->n_grp; ++g) free(st->grp[g].o_opt);
  free(st->grp);
  for (idx_t m = 0; m < st->tt.nmodes; ++m) mat_free(st->mats[m]);
  mat_free(st->mats[MAX_NMODES]);
  thd_free(st->thds, st->nthreads);
  free(st->opts);
  ref_free_tt(&st->tt);
  free(st);
}
