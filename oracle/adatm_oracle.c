/*
 * adatm_oracle.c -- CPU FP64 oracle for AdaTM's memoized MTTKRP sequence and
 * the CP-ALS sweep (hpcgarage/AdaTM, a patch over SPLATT v1.1.1).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for tests/, the smoke check and the
 * cpu_baseline leg of bench.py. The product library never links or calls it.
 *
 * Each function restates the reference algorithm and cites the reference
 * file:line it follows. Where the reference is defective (memo buffers never
 * re-zeroed, N=3 candidate-count UB, N-mode memo root with a partial memo at
 * begin_imten == N-1 that indexes leaf positions as fibers), the oracle
 * computes the mathematically defined result instead; those spots say so.
 *
 * SPLATT v1.1.1 is not vendored in the reference. Its pieces on the path
 * (tt_sort, mat_aTa, calc_gram_inv, mat_normalize, csf_frobsq,
 * cpd_post_process, the CSF mode orders) are restated from their documented
 * mathematics here; their parity is unpinned by any reference test.
 */
#include "adatm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#define ORC_ALLOC(T, n) ((T *)calloc((size_t)((n) > 0 ? (n) : 1), sizeof(T)))

static int orc_bitwidth(uint64_t v) {
  int b = 0;
  while (v) {
    ++b;
    v >>= 1;
  }
  return b;
}

/* Lexicographic order of the nonzeros by dim_perm: the effect of SPLATT's
 * tt_sort(tt, dim_perm[0], dim_perm) as called at adatm_rcsf.c:179 and
 * adatm_bench.c:179,222. Stable LSD counting sort over 16-bit digits, leaf
 * mode first, so equal coordinates keep their input order. */
void orc_sort_order(int nmodes, uint64_t nnz, const uint64_t *dims,
                    const uint64_t *inds, const uint64_t *perm,
                    uint64_t *order) {
  uint64_t *tmp = ORC_ALLOC(uint64_t, nnz);
  uint64_t *cnt = ORC_ALLOC(uint64_t, 65537);
  for (uint64_t i = 0; i < nnz; ++i) order[i] = i;
  for (int l = nmodes - 1; l >= 0; --l) {
    uint64_t const m = perm[l];
    const uint64_t *ind = inds + m * nnz;
    int const bits = orc_bitwidth(dims[m] > 0 ? dims[m] - 1 : 0);
    for (int sh = 0; sh < bits; sh += 16) {
      memset(cnt, 0, 65537 * sizeof(uint64_t));
      for (uint64_t i = 0; i < nnz; ++i) ++cnt[((ind[order[i]] >> sh) & 0xFFFF) + 1];
      for (int d = 0; d < 65536; ++d) cnt[d + 1] += cnt[d];
      for (uint64_t i = 0; i < nnz; ++i) {
        uint64_t const d = (ind[order[i]] >> sh) & 0xFFFF;
        tmp[cnt[d]++] = order[i];
      }
      memcpy(order, tmp, nnz * sizeof(uint64_t));
    }
  }
  free(cnt);
  free(tmp);
}

/* Input clean-up that precedes CSF construction: duplicates are summed in
 * FP64 in input order, then empty slices of every mode are compacted so that
 * slice s of the root maps to row s, the assumption behind fids[0] == NULL
 * (adatm_rcsf.c:51-56, mttkrp.c:334,811,877). Rewrites inds/vals/dims in
 * place, leaves the nonzeros in natural (mode 0..N-1) order, returns the new
 * nnz. */
uint64_t orc_coo_clean(int nmodes, uint64_t nnz, uint64_t *dims,
                       uint64_t *inds, double *vals) {
  uint64_t perm[ORC_MAXN] = {0};
  for (int m = 0; m < nmodes; ++m) perm[m] = (uint64_t)m;
  uint64_t *order = ORC_ALLOC(uint64_t, nnz);
  orc_sort_order(nmodes, nnz, dims, inds, perm, order);
  uint64_t *ninds = ORC_ALLOC(uint64_t, (uint64_t)nmodes * nnz);
  double *nvals = ORC_ALLOC(double, nnz);
  uint64_t out = 0;
  for (uint64_t i = 0; i < nnz; ++i) {
    uint64_t const src = order[i];
    int same = (out > 0);
    if (same) {
      for (int m = 0; m < nmodes && same; ++m)
        same = inds[(uint64_t)m * nnz + src] == ninds[(uint64_t)m * nnz + out - 1];
    }
    if (same) {
      nvals[out - 1] += vals[src];
    } else {
      for (int m = 0; m < nmodes; ++m)
        ninds[(uint64_t)m * nnz + out] = inds[(uint64_t)m * nnz + src];
      nvals[out] = vals[src];
      ++out;
    }
  }
  for (int m = 0; m < nmodes; ++m) {
    uint64_t *map = ORC_ALLOC(uint64_t, dims[m] + 1);
    for (uint64_t i = 0; i < out; ++i) map[ninds[(uint64_t)m * nnz + i]] = 1;
    uint64_t k = 0;
    for (uint64_t i = 0; i < dims[m]; ++i) {
      uint64_t const used = map[i];
      map[i] = k;
      k += used;
    }
    for (uint64_t i = 0; i < out; ++i)
      inds[(uint64_t)m * nnz + i] = map[ninds[(uint64_t)m * nnz + i]];
    dims[m] = k;
    free(map);
  }
  /* compact the mode-major layout from stride nnz to stride out */
  for (int m = 1; m < nmodes; ++m)
    memmove(inds + (uint64_t)m * out, inds + (uint64_t)m * nnz, out * sizeof(uint64_t));
  memcpy(vals, nvals, out * sizeof(double));
  free(ninds);
  free(nvals);
  free(order);
  return out;
}

/* Shared level builder. With fill == 0 it only counts fibers per level, as
 * count_nfibs does (adatm_rcsf.c:410-500); with fill != 0 it builds the CSF
 * arrays as p_csf_alloc_untiled does (adatm_rcsf.c:173-209): the root level
 * as p_mk_outerptr (adatm_rcsf.c:21-78), every further level as p_mk_fptr
 * (adatm_rcsf.c:93-163), including its in-place rewrite of the parent fptr
 * from nonzero positions to child-node positions (adatm_rcsf.c:147,161). */
static void orc_build_levels(orc_csf *ct, const uint64_t *inds,
                             const uint64_t *order, int fill) {
  int const N = ct->nmodes;
  uint64_t const nnz = ct->nnz;
  uint64_t *sl = ORC_ALLOC(uint64_t, nnz);
  ct->nfibs[N - 1] = nnz;
  if (nnz == 0) {
    for (int l = 0; l < N - 1; ++l) {
      ct->nfibs[l] = 0;
      if (fill) ct->fptr[l] = ORC_ALLOC(uint64_t, 1);
    }
    free(sl);
    return;
  }
  /* root level */
  {
    const uint64_t *ind = inds + ct->dim_perm[0] * nnz;
    for (uint64_t n = 0; n < nnz; ++n) sl[n] = ind[order[n]];
    uint64_t nf = 1;
    for (uint64_t x = 1; x < nnz; ++x)
      if (sl[x] != sl[x - 1]) ++nf;
    ct->nfibs[0] = nf;
    uint64_t *fp = ORC_ALLOC(uint64_t, nf + 1);
    uint64_t *ri = fill ? ORC_ALLOC(uint64_t, nf) : NULL;
    fp[0] = 0;
    if (ri) ri[0] = sl[0];
    uint64_t found = 1;
    for (uint64_t n = 1; n < nnz; ++n) {
      if (sl[n] != sl[n - 1]) {
        if (ri) ri[found] = sl[n];
        fp[found++] = n;
      }
    }
    fp[nf] = nnz;
    ct->fptr[0] = fp;
    ct->fids[0] = NULL;
    ct->root_ids = ri;
  }
  /* levels 1 .. N-2 */
  for (int l = 1; l < N - 1; ++l) {
    const uint64_t *ind = inds + ct->dim_perm[l] * nnz;
    for (uint64_t n = 0; n < nnz; ++n) sl[n] = ind[order[n]];
    uint64_t *fprev = ct->fptr[l - 1];
    uint64_t nf = 0;
    for (uint64_t s = 0; s < ct->nfibs[l - 1]; ++s) {
      ++nf;
      for (uint64_t f = fprev[s] + 1; f < fprev[s + 1]; ++f)
        if (sl[f] != sl[f - 1]) ++nf;
    }
    ct->nfibs[l] = nf;
    uint64_t *fp = ORC_ALLOC(uint64_t, nf + 1);
    uint64_t *fi = fill ? ORC_ALLOC(uint64_t, nf) : NULL;
    fp[0] = 0;
    uint64_t found = 0;
    for (uint64_t s = 0; s < ct->nfibs[l - 1]; ++s) {
      uint64_t const start = fprev[s] + 1;
      uint64_t const end = fprev[s + 1];
      fprev[s] = found;
      if (fi) fi[found] = sl[start - 1];
      fp[found++] = start - 1;
      for (uint64_t f = start; f < end; ++f) {
        if (sl[f] != sl[f - 1]) {
          if (fi) fi[found] = sl[f];
          fp[found++] = f;
        }
      }
    }
    fprev[ct->nfibs[l - 1]] = nf;
    fp[nf] = nnz;
    ct->fptr[l] = fp;
    ct->fids[l] = fi;
  }
  if (fill) {
    uint64_t *leaf = ORC_ALLOC(uint64_t, nnz);
    const uint64_t *ind = inds + ct->dim_perm[N - 1] * nnz;
    for (uint64_t n = 0; n < nnz; ++n) leaf[n] = ind[order[n]];
    ct->fids[N - 1] = leaf;
  }
  free(sl);
}

orc_csf *orc_csf_build(int nmodes, uint64_t nnz, const uint64_t *dims,
                       const uint64_t *inds, const double *vals,
                       const uint64_t *dim_perm) {
  orc_csf *ct = (orc_csf *)calloc(1, sizeof(orc_csf));
  ct->nmodes = nmodes;
  ct->nnz = nnz;
  for (int m = 0; m < nmodes; ++m) {
    ct->dims[m] = dims[m];
    ct->dim_perm[m] = dim_perm[m];
  }
  uint64_t *order = ORC_ALLOC(uint64_t, nnz);
  orc_sort_order(nmodes, nnz, dims, inds, dim_perm, order);
  ct->vals = ORC_ALLOC(double, nnz);
  for (uint64_t n = 0; n < nnz; ++n) ct->vals[n] = vals[order[n]];
  orc_build_levels(ct, inds, order, 1);
  free(order);
  return ct;
}

void orc_csf_free(orc_csf *ct) {
  if (!ct) return;
  for (int l = 0; l < ORC_MAXN; ++l) {
    free(ct->fptr[l]);
    free(ct->fids[l]);
  }
  free(ct->root_ids);
  free(ct->vals);
  free(ct);
}

void orc_count_nfibs(int nmodes, uint64_t nnz, const uint64_t *dims,
                     const uint64_t *inds, const uint64_t *o_opt,
                     uint64_t *nfibs) {
  orc_csf ct;
  memset(&ct, 0, sizeof(ct));
  ct.nmodes = nmodes;
  ct.nnz = nnz;
  for (int m = 0; m < nmodes; ++m) {
    ct.dims[m] = dims[m];
    ct.dim_perm[m] = o_opt[m];
  }
  uint64_t *order = ORC_ALLOC(uint64_t, nnz);
  orc_sort_order(nmodes, nnz, dims, inds, o_opt, order);
  orc_build_levels(&ct, inds, order, 0);
  for (int l = 0; l < nmodes; ++l) nfibs[l] = ct.nfibs[l];
  for (int l = 0; l < nmodes; ++l) {
    free(ct.fptr[l]);
    free(ct.fids[l]);
  }
  free(ct.root_ids);
  free(order);
}

/* SPLATT's plain CSF mode orders (SPLATT's csf.c is absent from the
 * reference; the order used here is the definition this project adopts):
 * which == 0 (ONEMODE): all modes by dimension ascending, ties by mode id;
 * which == 1 (root-first, used by TWOMODE's second tensor and ALLMODE):
 * `root` first, then the other modes by dimension ascending. */
void orc_splatt_perm(int nmodes, const uint64_t *dims, int which,
                     uint64_t root, uint64_t *perm) {
  int k = 0;
  if (which == 1) perm[k++] = root;
  for (int pass = 0; pass < nmodes; ++pass) {
    /* selection by (dim, mode) ascending keeps the order total */
    uint64_t best = (uint64_t)-1;
    for (int m = 0; m < nmodes; ++m) {
      if (which == 1 && (uint64_t)m == root) continue;
      int taken = 0;
      for (int j = 0; j < k; ++j) taken |= (perm[j] == (uint64_t)m);
      if (taken) continue;
      if (best == (uint64_t)-1 || dims[m] < dims[best]) best = (uint64_t)m;
    }
    if (best == (uint64_t)-1) break;
    perm[k++] = best;
  }
}

/* ------------------------------------------------------------------------ */
/* planner                                                                   */
/* ------------------------------------------------------------------------ */

/* argmin_elem_range (adatm_utils.c:33-51): first index of the smallest entry
 * greater than `con`. Returns n when there is none (undefined in the
 * reference). */
static uint64_t orc_argmin_range(const uint64_t *arr, uint64_t n, uint64_t con) {
  uint64_t mkr = n;
  for (uint64_t i = 0; i < n; ++i)
    if (arr[i] > con) {
      mkr = i;
      break;
    }
  if (mkr == n) return n;
  for (uint64_t i = 0; i < n; ++i)
    if (arr[i] > con && arr[i] < arr[mkr]) mkr = i;
  return mkr;
}

/* array_min_range (adatm_utils.c:80-97): smallest entry greater than `con`.
 * Returns 0 when there is none; the reference reads an uninitialised value
 * there (its N=3 candidate count, adatm_bench.c:303-326). */
static uint64_t orc_min_range(const uint64_t *arr, uint64_t n, uint64_t con) {
  int found = 0;
  uint64_t mkr = 0;
  for (uint64_t i = 0; i < n; ++i)
    if (arr[i] > con) {
      mkr = arr[i];
      found = 1;
      break;
    }
  if (!found) return 0;
  for (uint64_t i = 0; i < n; ++i)
    if (arr[i] > con && arr[i] < mkr) mkr = arr[i];
  return mkr;
}

/* pair_sort / pair_sort_range (adatm_sort.c:10-75): the reference's own
 * quicksort of (mode, dim) pairs by dim. Its steps are kept so that equal
 * dims come out in the same order as the reference's o_opt. */
static void orc_pair_sort_range(uint64_t *x, uint64_t *y, uint64_t start,
                                uint64_t end) {
  uint64_t i = start + 1;
  uint64_t j = end - 1;
  uint64_t const k = start + ((end - start) / 2);
  uint64_t const px = x[k], py = y[k];
  x[k] = x[start];
  y[k] = y[start];
  while (i < j) {
    if (py < y[i]) {
      if (py > y[j]) {
        uint64_t t = x[i];
        x[i] = x[j];
        x[j] = t;
        t = y[i];
        y[i] = y[j];
        y[j] = t;
        ++i;
      }
      --j;
    } else {
      if (py < y[j]) --j;
      ++i;
    }
  }
  if (py < y[i]) --i;
  x[start] = x[i];
  x[i] = px;
  y[start] = y[i];
  y[i] = py;
  if (i > start + 1) orc_pair_sort_range(x, y, start, i);
  ++i;
  if (end - i > 1) orc_pair_sort_range(x, y, i, end);
}

void orc_pair_sort(uint64_t *x, uint64_t *y, uint64_t n) {
  if (n > 1) orc_pair_sort_range(x, y, 0, n);
}

/* decide_product_order (adatm_bench.c:62-74) and decide_candidate_configs
 * (adatm_bench.c:276-458). Returns the number of configurations written. */
int orc_candidate_configs(int nmodes, const uint64_t *dims,
                          orc_config *configs, int max_configs) {
  uint64_t const N = (uint64_t)nmodes;
  uint64_t po[ORC_MAXN][2 * ORC_MAXN];
  memset(po, 0, sizeof(po));
  for (uint64_t m = 0; m < N; ++m) {
    for (uint64_t i = m + 1; i < N; ++i) po[m][i] = 1;
    for (uint64_t i = 0; i < m; ++i) po[m][i + N] = 1;
  }
  uint64_t const n_grp_cal = (uint64_t)ceil((double)N / sqrt(2.0 * (double)(N - 1)));
  uint64_t maxn[ORC_MAXN + 2], begin[ORC_MAXN + 2], memo[ORC_MAXN + 2];
  int cfg = 0;
  for (uint64_t ng = 0; ng < n_grp_cal + 1; ++ng) {
    uint64_t n_grp = ng + 1;
    uint64_t const aver = N / n_grp;
    uint64_t rest = N % n_grp;
    if (aver == 1 && rest > 0) continue;
    if (n_grp >= N) continue;
    memset(maxn, 0, sizeof(maxn));
    memset(begin, 0, sizeof(begin));
    memset(memo, 0, sizeof(memo));
    if (n_grp != 1) {
      for (uint64_t g = 0; g < n_grp; ++g) {
        if (rest > 0) {
          maxn[g] = aver;
          --rest;
        } else {
          maxn[g] = aver - 1;
        }
        begin[g] = maxn[g] + 1;
      }
      memo[0] = 0;
      for (uint64_t g = 1; g < n_grp; ++g) memo[g] = memo[g - 1] + maxn[g - 1] + 1;
    } else {
      maxn[0] = N - 2;
      maxn[1] = 0;
      begin[0] = N - 1;
      begin[1] = 1;
      memo[0] = 0;
      memo[1] = N - 1;
      n_grp = 2;
    }
    uint64_t const mm = orc_min_range(maxn, n_grp_cal + 1, 0);
    for (uint64_t i = 0; i < mm; ++i) {
      if (cfg >= max_configs) return cfg;
      orc_config *c = configs + cfg;
      memset(c, 0, sizeof(*c));
      c->n_grp = n_grp;
      for (uint64_t g = 0; g < n_grp; ++g) {
        orc_grp *gp = c->grp + g;
        gp->memo_mode = memo[g];
        gp->begin_imten = begin[g];
        gp->n_imten = (memo[g] != N - 1) ? maxn[g] - i : 0;
        uint64_t const mmode = memo[g];
        uint64_t sum_times[2 * ORC_MAXN], tmp_times[2 * ORC_MAXN], tmp_opt[ORC_MAXN];
        memset(sum_times, 0, sizeof(sum_times));
        memset(tmp_times, 0, sizeof(tmp_times));
        memset(tmp_opt, 0, sizeof(tmp_opt));
        gp->o_opt[0] = mmode;
        tmp_opt[0] = mmode;
        for (uint64_t j = mmode; j <= mmode + maxn[g]; ++j)
          for (uint64_t k = 0; k < 2 * N; ++k) sum_times[k] += po[j][k];
        for (uint64_t k = 0; k < 2 * N; ++k)
          if (po[mmode][k] > 0) tmp_times[k] = sum_times[k];
        for (uint64_t j = 1; j < N; ++j) {
          uint64_t t = orc_argmin_range(tmp_times, 2 * N, 0);
          tmp_times[t] = 0;
          if (t >= N) t -= N;
          tmp_opt[j] = t;
        }
        uint64_t const ss = N - gp->begin_imten;
        uint64_t px[ORC_MAXN], py[ORC_MAXN];
        for (uint64_t j = 0; j < ss; ++j) {
          px[j] = tmp_opt[j + gp->begin_imten];
          py[j] = dims[px[j]];
        }
        orc_pair_sort(px, py, ss);
        for (uint64_t j = 0; j < ss; ++j) gp->o_opt[j + gp->begin_imten] = px[j];
        for (uint64_t j = 1; j < gp->begin_imten; ++j) gp->o_opt[j] = tmp_opt[j];
      }
      ++cfg;
    }
  }
  return cfg;
}

/* predict_csf_bytes_adaptive (adatm_rcsf.c:329-345) */
static uint64_t orc_pcsf_bytes(int N, uint64_t nnz, const uint64_t *nf) {
  uint64_t b = nnz * 8 + nnz * 8;
  for (int m = 0; m < N - 1; ++m) b += (nf[m] + 1) * 8 + nf[m] * 8;
  return b;
}
/* predict_rcsf_bytes_adaptive (adatm_rcsf.c:347-363) */
static uint64_t orc_prcsf_bytes(uint64_t R, uint64_t begin, uint64_t n_imten,
                                const uint64_t *nf) {
  uint64_t b = 0;
  for (uint64_t i = 0; i < n_imten; ++i) b += nf[begin - i] * R * 8;
  return b;
}
/* predict_csf_ops_adaptive (adatm_rcsf.c:365-379) */
static uint64_t orc_pcsf_ops(int N, uint64_t R, const uint64_t *nf) {
  uint64_t ops = 0;
  for (int m = N; m >= 1; --m) ops += nf[m - 1] * R * 2;
  return ops;
}
/* predict_rcsf_ops_adaptive (adatm_rcsf.c:382-406) */
static uint64_t orc_prcsf_ops(uint64_t R, uint64_t begin, uint64_t n_imten,
                              uint64_t num_re, const uint64_t *nf) {
  uint64_t ops = 0;
  if (n_imten == 0) return 0;
  uint64_t const end = begin - n_imten + 1;
  for (uint64_t i = 1; i <= num_re; ++i) {
    if (i < end)
      ops += nf[end - 1] * R * 2;
    else if (i < begin)
      ops += nf[i] * R * 2;
  }
  return ops;
}

/* predict_candidates_adaptive (adatm_bench.c:145-272). Fiber counts are
 * recomputed only when n_grp changes; configurations that share n_grp with
 * the previous one reuse the fiber counts of the LAST group counted for
 * every group (adatm_bench.c:246-261). That behaviour decides which plan the
 * reference picks, so it is kept. */
void orc_predict_candidates(int nmodes, uint64_t nnz, const uint64_t *dims,
                            const uint64_t *inds, uint64_t nfactors,
                            orc_config *configs, int nconfigs) {
  uint64_t const N = (uint64_t)nmodes;
  uint64_t grp_nfibs[ORC_MAXN][ORC_MAXN];
  memset(grp_nfibs, 0, sizeof(grp_nfibs));
  uint64_t cur = 0; /* which grp_nfibs row nfibs_per_grp points at */
  uint64_t num_re = 0;
  uint64_t csf_bytes = 0, rcsf_bytes = 0, csf_ops = 0, rcsf_ops = 0;
  uint64_t old_n_grp = 0;
  for (int c = 0; c < nconfigs; ++c) {
    orc_config *cf = configs + c;
    uint64_t const n_grp = cf->n_grp;
    rcsf_bytes = 0;
    rcsf_ops = 0;
    int const recount = (c == 0) || (n_grp != old_n_grp);
    if (recount) {
      old_n_grp = n_grp;
      csf_bytes = 0;
      csf_ops = 0;
    }
    for (uint64_t g = 0; g < n_grp; ++g) {
      orc_grp const *gp = cf->grp + g;
      if (recount) {
        cur = gp->memo_mode;
        uint64_t *nf = grp_nfibs[cur];
        memset(nf, 0, sizeof(grp_nfibs[0]));
        orc_count_nfibs(nmodes, nnz, dims, inds, gp->o_opt, nf);
        nf[N - 1] = nnz;
      }
      if (gp->n_imten != 0) {
        if (g < n_grp - 1)
          num_re = cf->grp[g + 1].memo_mode - gp->memo_mode - 1;
        else
          num_re = N - gp->memo_mode - 1;
      }
      uint64_t const *nf = grp_nfibs[cur];
      if (recount) {
        csf_bytes += orc_pcsf_bytes(nmodes, nnz, nf);
        csf_ops += orc_pcsf_ops(nmodes, nfactors, nf);
      }
      rcsf_bytes += orc_prcsf_bytes(nfactors, gp->begin_imten, gp->n_imten, nf);
      rcsf_ops += orc_prcsf_ops(nfactors, gp->begin_imten, gp->n_imten, num_re, nf);
    }
    cf->pspace = csf_bytes + rcsf_bytes;
    cf->pops = csf_ops + rcsf_ops;
  }
}

/* limit_candidates_by_space (adatm_bench.c:77-105) followed by
 * choose_candidates_by_strategy (adatm_bench.c:108-142). The reference
 * returns a position in the space-filtered list and decide_parameters_auto
 * then indexes the unfiltered list with it (adatm_bench.c:482-485); that is
 * kept. Returns -1 when no configuration fits (undefined in the reference). */
int orc_choose_config(const orc_config *configs, int nconfigs, int strategy,
                      double slimit) {
  int real[4 * ORC_MAXN * ORC_MAXN];
  int nreal = 0;
  for (int c = 0; c < nconfigs; ++c)
    if ((double)configs[c].pspace < slimit) real[nreal++] = c;
  if (nreal == 0) return -1;
  int opt = 0;
  uint64_t min_ops = configs[real[0]].pops;
  uint64_t min_space = configs[real[0]].pspace;
  for (int c = 1; c < nreal; ++c) {
    orc_config const *cf = configs + real[c];
    if (strategy == 1 && cf->pops < min_ops) {
      min_ops = cf->pops;
      opt = c;
    } else if (strategy == 2 && cf->pspace < min_space) {
      min_space = cf->pspace;
      opt = c;
    }
  }
  return opt;
}

/* decide_parameters_auto (adatm_bench.c:462-508) with SLIMIT = 90e9 bytes
 * (adatm_base.h:4). */
uint64_t orc_plan(int nmodes, uint64_t nnz, const uint64_t *dims,
                  const uint64_t *inds, uint64_t nfactors, int strategy,
                  orc_grp *grp_out, orc_config *all_out, int *nconfigs_out) {
  orc_config configs[4 * ORC_MAXN];
  int const n = orc_candidate_configs(nmodes, dims, configs, 4 * ORC_MAXN);
  orc_predict_candidates(nmodes, nnz, dims, inds, nfactors, configs, n);
  int const opt = orc_choose_config(configs, n, strategy, 90000000000.0);
  if (all_out)
    for (int c = 0; c < n; ++c) all_out[c] = configs[c];
  if (nconfigs_out) *nconfigs_out = n;
  if (opt < 0) return 0;
  for (uint64_t g = 0; g < configs[opt].n_grp; ++g) grp_out[g] = configs[opt].grp[g];
  return configs[opt].n_grp;
}

/* locate_ind_special (adatm_utils.c:9-30), including its unconditional
 * break after the first loop iteration. */
static double orc_locate_special(const uint64_t *arr, uint64_t len, uint64_t ele,
                                 uint64_t nmodes) {
  double loc = -1;
  if (arr[0] == ele) loc = 0;
  for (uint64_t i = 1; i < len; ++i) {
    if (arr[i] == ele)
      loc = (double)i;
    else if (arr[i - 1] < ele && ele < arr[i])
      loc = (double)i - 0.5;
    break;
  }
  if (arr[len - 1] < ele && ele < nmodes) loc = (double)len - 0.5;
  return loc;
}

/* decide_use_csfs (mttkrp.c:1940-2033). Tag 0: memo root, 1: reuse,
 * 2: recompute as an internal or leaf MTTKRP. */
void orc_decide_use_csfs(int nmodes, const orc_grp *grp, uint64_t n_grp,
                         uint64_t n_csf, uint64_t *use_csfs,
                         uint64_t *use_tags) {
  uint64_t const N = (uint64_t)nmodes;
  uint64_t gm[ORC_MAXN];
  for (uint64_t m = 0; m < N; ++m) use_tags[m] = 0;
  for (uint64_t g = 0; g < n_grp; ++g) gm[g] = grp[g].memo_mode;
  if (n_csf == n_grp) {
    for (uint64_t g = 0; g + 1 < n_grp; ++g) {
      uint64_t const mode = gm[g];
      use_csfs[mode] = g;
      use_tags[mode] = 0;
      for (uint64_t rm = mode + 1; rm < gm[g + 1]; ++rm) {
        use_csfs[rm] = g;
        use_tags[rm] = 1;
      }
    }
    uint64_t const mode = gm[n_grp - 1];
    use_csfs[mode] = n_grp - 1;
    use_tags[mode] = 0;
    for (uint64_t rm = mode + 1; rm < N; ++rm) {
      use_csfs[rm] = n_grp - 1;
      use_tags[rm] = 1;
    }
    return;
  }
  uint64_t csf_modes[ORC_MAXN];
  uint64_t ci = 0;
  for (uint64_t g = 0; g < n_grp; ++g)
    if (grp[g].n_imten > 0) csf_modes[ci++] = grp[g].memo_mode;
  for (uint64_t g = 0; g + 1 < n_grp; ++g) {
    for (int pass = 0; pass < 2; ++pass) {
      uint64_t const mode = pass == 0 ? gm[g] : gm[n_grp - 1];
      uint64_t const stop = pass == 0 ? gm[g + 1] : N;
      double const loc = orc_locate_special(csf_modes, n_csf, mode, N);
      if (loc < 0) continue;
      uint64_t const il = (uint64_t)loc;
      uint64_t const tag = (loc - (double)il == 0) ? 0 : 2;
      use_csfs[mode] = il;
      use_tags[mode] = tag;
      for (uint64_t rm = mode + 1; rm < stop; ++rm) {
        use_csfs[rm] = il;
        use_tags[rm] = tag == 0 ? 1 : 2;
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* MTTKRP                                                                    */
/* ------------------------------------------------------------------------ */

static uint64_t orc_depth(const orc_csf *ct, uint64_t mode) {
  for (int l = 0; l < ct->nmodes; ++l)
    if (ct->dim_perm[l] == mode) return (uint64_t)l;
  return (uint64_t)ct->nmodes;
}

/* Bottom-up contraction of the tree from level `src` (the leaf nonzeros when
 * src_vals == NULL, else the dense node rows src_vals of level src) up to
 * level `top`. Level l's node value is the sum over its children c of
 * value(c) * U_{dim_perm[l+1]}[fids[l+1][c]]; at the leaf the children are the
 * nonzeros and value(c) is the nonzero. This is p_spttm (mttkrp.c:891-928)
 * followed by the p_spt2t_add_hada chain (mttkrp.c:828-853), and the per-slice
 * DFS p_propagate_up (mttkrp.c:241-304) / p_propagate_up_reuse
 * (mttkrp.c:169-236) computes the same node sums. store[l] (if non-NULL)
 * receives level l's rows. Returns a malloc'd F_top x R array. */
static double *orc_contract(const orc_csf *ct, double *const *mats, uint64_t R,
                            int src, const double *src_vals, int top,
                            double *const *store) {
  int const N = ct->nmodes;
  double *cur;
  int lev;
  if (src_vals == NULL) {
    lev = N - 2;
    uint64_t const F = ct->nfibs[lev];
    cur = ORC_ALLOC(double, F * R);
    const double *U = mats[ct->dim_perm[N - 1]];
    for (uint64_t f = 0; f < F; ++f) {
      double *o = cur + f * R;
      for (uint64_t j = ct->fptr[lev][f]; j < ct->fptr[lev][f + 1]; ++j) {
        double const v = ct->vals[j];
        const double *row = U + ct->fids[N - 1][j] * R;
        for (uint64_t r = 0; r < R; ++r) o[r] += v * row[r];
      }
    }
  } else {
    lev = src;
    uint64_t const F = ct->nfibs[lev];
    cur = ORC_ALLOC(double, F * R);
    memcpy(cur, src_vals, F * R * sizeof(double));
  }
  if (store && store[lev] && src_vals == NULL)
    memcpy(store[lev], cur, ct->nfibs[lev] * R * sizeof(double));
  while (lev > top) {
    uint64_t const F = ct->nfibs[lev - 1];
    double *nxt = ORC_ALLOC(double, F * R);
    const double *U = mats[ct->dim_perm[lev]];
    for (uint64_t s = 0; s < F; ++s) {
      double *o = nxt + s * R;
      for (uint64_t f = ct->fptr[lev - 1][s]; f < ct->fptr[lev - 1][s + 1]; ++f) {
        const double *in = cur + f * R;
        const double *row = U + ct->fids[lev][f] * R;
        for (uint64_t r = 0; r < R; ++r) o[r] += in[r] * row[r];
      }
    }
    free(cur);
    cur = nxt;
    --lev;
    if (store && store[lev]) memcpy(store[lev], cur, F * R * sizeof(double));
  }
  return cur;
}

/* Top-down prefix products: P_l[node] = U_{perm[0]}[root id] * ... *
 * U_{perm[l]}[fids[l][node]], the buf[] chain that the internal/leaf/reuse
 * kernels push down with p_assign_hada (mttkrp.c:1500-1505, 1283-1288,
 * 1641-1647). Returns a malloc'd F_l x R array. */
static double *orc_prefix(const orc_csf *ct, double *const *mats, uint64_t R,
                          int lvl) {
  uint64_t F = ct->nfibs[0];
  double *cur = ORC_ALLOC(double, F * R);
  const double *U0 = mats[ct->dim_perm[0]];
  for (uint64_t s = 0; s < F; ++s)
    memcpy(cur + s * R, U0 + ct->root_ids[s] * R, R * sizeof(double));
  for (int l = 1; l <= lvl; ++l) {
    uint64_t const Fl = ct->nfibs[l];
    double *nxt = ORC_ALLOC(double, Fl * R);
    const double *U = mats[ct->dim_perm[l]];
    for (uint64_t p = 0; p < ct->nfibs[l - 1]; ++p)
      for (uint64_t f = ct->fptr[l - 1][p]; f < ct->fptr[l - 1][p + 1]; ++f)
        for (uint64_t r = 0; r < R; ++r)
          nxt[f * R + r] = cur[p * R + r] * U[ct->fids[l][f] * R + r];
    free(cur);
    cur = nxt;
  }
  return cur;
}

/* Scatter node sums of level d into the output rows fids[d]:
 * out[fids[d][y]] += S_d[y] * P_{d-1}[parent(y)] (mttkrp.c:1533-1536,
 * 1660-1668, 640-644); for d == 0 the root rows take S_0 directly
 * (mttkrp.c:818-822, 877-885). */
static void orc_scatter(const orc_csf *ct, double *const *mats, uint64_t R,
                        int d, const double *S, double *out) {
  if (d == 0) {
    for (uint64_t s = 0; s < ct->nfibs[0]; ++s)
      for (uint64_t r = 0; r < R; ++r) out[ct->root_ids[s] * R + r] += S[s * R + r];
    return;
  }
  double *P = orc_prefix(ct, mats, R, d - 1);
  for (uint64_t p = 0; p < ct->nfibs[d - 1]; ++p)
    for (uint64_t y = ct->fptr[d - 1][p]; y < ct->fptr[d - 1][p + 1]; ++y) {
      double *o = out + ct->fids[d][y] * R;
      for (uint64_t r = 0; r < R; ++r) o[r] += S[y * R + r] * P[p * R + r];
    }
  free(P);
}

/* Plain CSF MTTKRP for `mode` of one tree: root (p_csf_mttkrp_root,
 * mttkrp.c:766-825; root3 :367-425), internal (p_csf_mttkrp_internal,
 * mttkrp.c:1452-1540; internal3 :534-597) or leaf (p_csf_mttkrp_leaf,
 * mttkrp.c:1219-1300; leaf3 :650-705). Accumulates into out. */
static void orc_mttkrp_tree(const orc_csf *ct, double *const *mats,
                            uint64_t mode, uint64_t R, double *out) {
  int const N = ct->nmodes;
  int const d = (int)orc_depth(ct, mode);
  if (ct->nnz == 0) return;
  if (d == N - 1) {
    double *P = orc_prefix(ct, mats, R, N - 2);
    for (uint64_t f = 0; f < ct->nfibs[N - 2]; ++f)
      for (uint64_t j = ct->fptr[N - 2][f]; j < ct->fptr[N - 2][f + 1]; ++j) {
        double *o = out + ct->fids[N - 1][j] * R;
        for (uint64_t r = 0; r < R; ++r) o[r] += ct->vals[j] * P[f * R + r];
      }
    free(P);
    return;
  }
  double *S = orc_contract(ct, mats, R, N - 1, NULL, d, NULL);
  orc_scatter(ct, mats, R, d, S, out);
  free(S);
}

void orc_mttkrp_csf(const orc_csf *ct, double *const *mats, uint64_t mode,
                    uint64_t nfactors, double *out) {
  memset(out, 0, ct->dims[mode] * nfactors * sizeof(double));
  orc_mttkrp_tree(ct, mats, mode, nfactors, out);
}

orc_model *orc_model_build(int nmodes, uint64_t nnz, const uint64_t *dims,
                           const uint64_t *inds, const double *vals,
                           uint64_t nfactors, uint64_t n_grp,
                           const orc_grp *grp) {
  orc_model *md = (orc_model *)calloc(1, sizeof(orc_model));
  md->nmodes = nmodes;
  md->nfactors = nfactors;
  for (int m = 0; m < nmodes; ++m) md->dims[m] = dims[m];
  md->n_grp = n_grp;
  for (uint64_t g = 0; g < n_grp; ++g) md->grp[g] = grp[g];
  /* csf_alloc_adaptive, TIME_EFFICIENT (adatm_rcsf.c:503-527): one CSF per
   * group, rooted at o_opt order. */
  md->n_csf = n_grp;
  for (uint64_t g = 0; g < n_grp; ++g)
    md->csf[g] = orc_csf_build(nmodes, nnz, dims, inds, vals, grp[g].o_opt);
  /* rcsf_alloc_adaptive / p_rcsf_alloc_untiled_adaptive
   * (adatm_rcsf.c:216-278,591-615): memo tree deg stores
   * nfibs[begin_imten-1-deg] x R values. */
  for (uint64_t g = 0; g < n_grp; ++g) {
    for (uint64_t deg = 0; deg < grp[g].n_imten; ++deg) {
      uint64_t const lvl = grp[g].begin_imten - 1 - deg;
      md->memo_rows[g][deg] = md->csf[g]->nfibs[lvl];
      md->memo[g][deg] = ORC_ALLOC(double, md->memo_rows[g][deg] * nfactors);
    }
  }
  orc_decide_use_csfs(nmodes, grp, n_grp, md->n_csf, md->use_csfs, md->use_tags);
  return md;
}

void orc_model_free(orc_model *md) {
  if (!md) return;
  for (uint64_t g = 0; g < md->n_csf; ++g) orc_csf_free(md->csf[g]);
  for (int g = 0; g < ORC_MAXN; ++g)
    for (int d = 0; d < ORC_MAXN; ++d) free(md->memo[g][d]);
  free(md);
}

/* mttkrp_csf_adaptive (mttkrp.c:2037-2090). Tag 0 with a memo plan is the
 * memo root (p_csf_mttkrp_root_genreuse_adaptive, mttkrp.c:934-1079;
 * p_csf_mttkrp_root3_reuse_adaptive, mttkrp.c:429-531): it overwrites memo
 * tree deg with the level (begin_imten-1-deg) node sums on every call (the
 * reference accumulates into buffers it never re-zeroes, mttkrp.c:922,848).
 * Tag 1 is the reuse MTTKRP (p_csf_mttkrp_internal_reuse_adaptive,
 * mttkrp.c:1547-1682; internal3_reuse :599-647): it starts from memo tree
 * indeg-1, where indeg counts the leading stored levels that lie below the
 * output level (mttkrp.c:1578-1588 with rcsf_reverse_mode_order,
 * adatm_rcsf.c:313-326). Tag 2 recomputes with the plain CSF kernels. */
void orc_mttkrp_adaptive(orc_model *md, double *const *mats, uint64_t mode,
                         double *out) {
  uint64_t const R = md->nfactors;
  memset(out, 0, md->dims[mode] * R * sizeof(double));
  uint64_t const g = md->use_csfs[mode];
  uint64_t const tag = md->use_tags[mode];
  orc_csf const *ct = md->csf[g];
  orc_grp const *gp = md->grp + g;
  int const N = ct->nmodes;
  if (ct->nnz == 0) return;
  if (tag == 0) {
    if (gp->n_imten == 0) {
      orc_mttkrp_tree(ct, mats, mode, R, out);
      return;
    }
    double *store[ORC_MAXN];
    memset(store, 0, sizeof(store));
    for (uint64_t deg = 0; deg < gp->n_imten; ++deg)
      store[gp->begin_imten - 1 - deg] = md->memo[g][deg];
    double *S = orc_contract(ct, mats, R, N - 1, NULL, 0, store);
    orc_scatter(ct, mats, R, 0, S, out);
    free(S);
  } else if (tag == 1) {
    uint64_t const d = orc_depth(ct, mode);
    uint64_t const b = gp->begin_imten;
    uint64_t rd[ORC_MAXN];
    uint64_t j = 0;
    for (int64_t i = (int64_t)b; i >= 0; --i)
      if ((uint64_t)i != d) rd[j++] = (uint64_t)i;
    uint64_t indeg = 0;
    for (uint64_t i = 0; i < gp->n_imten; ++i)
      if (b - i == rd[i]) ++indeg;
    if (indeg == 0) return;
    int const L = (int)(b - indeg);
    double *S = orc_contract(ct, mats, R, L, md->memo[g][indeg - 1], (int)d, NULL);
    orc_scatter(ct, mats, R, (int)d, S, out);
    free(S);
  } else {
    orc_mttkrp_tree(ct, mats, mode, R, out);
  }
}

/* ------------------------------------------------------------------------ */
/* CP-ALS                                                                    */
/* ------------------------------------------------------------------------ */

static uint64_t orc_mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

/* Seeded factor initialisation, uniform in [0,1): entry (i, r) of mode m is
 * mix64(mix64(seed * 0x100000001B3 + m) + i * R + r) >> 11, scaled by 2^-53.
 * Stands in for SPLATT's mat_rand (adatm_cpd.c:227-229), whose generator is
 * not part of the reference. */
void orc_factor_init(uint64_t seed, uint64_t mode, uint64_t rows,
                     uint64_t nfactors, double *out) {
  uint64_t const key = orc_mix64(seed * 0x100000001B3ull + mode);
  for (uint64_t x = 0; x < rows * nfactors; ++x)
    out[x] = (double)(orc_mix64(key + x) >> 11) * (1.0 / 9007199254740992.0);
}

/* mat_aTa: G = A^T A (SPLATT, called at adatm_cpd.c:288,335). */
static void orc_ata(const double *A, uint64_t I, uint64_t R, double *G) {
  memset(G, 0, R * R * sizeof(double));
  for (uint64_t i = 0; i < I; ++i)
    for (uint64_t a = 0; a < R; ++a)
      for (uint64_t b = 0; b < R; ++b) G[a * R + b] += A[i * R + a] * A[i * R + b];
}

/* calc_gram_inv (SPLATT, called at adatm_cpd.c:321): the Hadamard product of
 * every Gram matrix but `mode`, inverted through its Cholesky factor. */
static void orc_gram_inv(double *const *G, int nmodes, uint64_t mode, uint64_t R,
                         double *Vinv) {
  double *V = ORC_ALLOC(double, R * R);
  double *L = ORC_ALLOC(double, R * R);
  for (uint64_t x = 0; x < R * R; ++x) V[x] = 1.0;
  for (int m = 0; m < nmodes; ++m) {
    if ((uint64_t)m == mode) continue;
    for (uint64_t x = 0; x < R * R; ++x) V[x] *= G[m][x];
  }
  for (uint64_t j = 0; j < R; ++j) {
    double s = V[j * R + j];
    for (uint64_t k = 0; k < j; ++k) s -= L[j * R + k] * L[j * R + k];
    L[j * R + j] = sqrt(s);
    for (uint64_t i = j + 1; i < R; ++i) {
      double t = V[i * R + j];
      for (uint64_t k = 0; k < j; ++k) t -= L[i * R + k] * L[j * R + k];
      L[i * R + j] = t / L[j * R + j];
    }
  }
  /* solve L Y = I, then L^T X = Y, one column at a time */
  double *y = ORC_ALLOC(double, R);
  for (uint64_t c = 0; c < R; ++c) {
    for (uint64_t i = 0; i < R; ++i) {
      double t = (i == c) ? 1.0 : 0.0;
      for (uint64_t k = 0; k < i; ++k) t -= L[i * R + k] * y[k];
      y[i] = t / L[i * R + i];
    }
    for (int64_t i = (int64_t)R - 1; i >= 0; --i) {
      double t = y[i];
      for (uint64_t k = (uint64_t)i + 1; k < R; ++k) t -= L[k * R + (uint64_t)i] * Vinv[k * R + c];
      Vinv[(uint64_t)i * R + c] = t / L[(uint64_t)i * R + (uint64_t)i];
    }
  }
  free(y);
  free(L);
  free(V);
}

/* mat_normalize (SPLATT, adatm_cpd.c:328-332): which == 2 gives column
 * 2-norms; which == 0 gives column maxima floored at 1 (the max starts from
 * 0 and takes signed values). Columns are divided by lambda. */
static void orc_normalize(double *A, uint64_t I, uint64_t R, double *lambda,
                          int which) {
  for (uint64_t r = 0; r < R; ++r) lambda[r] = 0;
  if (which == 2) {
    for (uint64_t i = 0; i < I; ++i)
      for (uint64_t r = 0; r < R; ++r) lambda[r] += A[i * R + r] * A[i * R + r];
    for (uint64_t r = 0; r < R; ++r) lambda[r] = sqrt(lambda[r]);
  } else {
    for (uint64_t i = 0; i < I; ++i)
      for (uint64_t r = 0; r < R; ++r)
        if (A[i * R + r] > lambda[r]) lambda[r] = A[i * R + r];
    for (uint64_t r = 0; r < R; ++r)
      if (lambda[r] < 1.0) lambda[r] = 1.0;
  }
  for (uint64_t i = 0; i < I; ++i)
    for (uint64_t r = 0; r < R; ++r) A[i * R + r] /= lambda[r];
}

/* MTTKRP of one mode through a caller-chosen method (the memoized model,
 * a plain tree per mode, or the COO loop below). */
typedef void (*orc_mttkrp_fn)(void *ctx, double *const *mats, uint64_t mode, double *out);

typedef struct orc_plain_ctx {
  const orc_csf *const *csfs;
  uint64_t R;
} orc_plain_ctx;

static void orc_mttkrp_model_cb(void *ctx, double *const *mats, uint64_t mode, double *out) {
  orc_mttkrp_adaptive((orc_model *)ctx, mats, mode, out);
}

static void orc_mttkrp_plain_cb(void *ctx, double *const *mats, uint64_t mode, double *out) {
  orc_plain_ctx const *p = (orc_plain_ctx const *)ctx;
  orc_mttkrp_csf(p->csfs[mode], mats, mode, p->R, out);
}

/* cpd_als_iterate_adaptive (adatm_cpd.c:256-373) with p_calc_fit
 * (adatm_cpd.c:179-200), p_kruskal_norm (:59-90) and p_tt_kruskal_inner
 * (:109-160), followed by cpd_post_process (SPLATT, :364): every factor is
 * 2-normalised and lambda absorbs the norms. The MTTKRP of each mode comes
 * from `mttkrp`. mats[m] (dims[m] x R, row-major) hold the initial factors
 * on entry and the final factors on return. Returns the last fit. */
static double orc_als_core(int N, const uint64_t *dims, double ttnormsq, uint64_t R,
                           orc_mttkrp_fn mttkrp, void *ctx, double *const *mats,
                           double *lambda, uint64_t niters, double tol,
                           double *fit_trace, uint64_t *iters_done) {
  uint64_t maxdim = 0;
  for (int m = 0; m < N; ++m)
    if (dims[m] > maxdim) maxdim = dims[m];
  double *G[ORC_MAXN];
  for (int m = 0; m < N; ++m) {
    G[m] = ORC_ALLOC(double, R * R);
    orc_ata(mats[m], dims[m], R, G[m]);
  }
  double *Vinv = ORC_ALLOC(double, R * R);
  double *M = ORC_ALLOC(double, maxdim * R);
  double fit = 0, oldfit = 0;
  uint64_t it = 0;
  for (it = 0; it < niters; ++it) {
    for (int m = 0; m < N; ++m) {
      uint64_t const I = dims[m];
      mttkrp(ctx, mats, (uint64_t)m, M);
      orc_gram_inv(G, N, (uint64_t)m, R, Vinv);
      double *A = mats[m];
      for (uint64_t i = 0; i < I; ++i)
        for (uint64_t r = 0; r < R; ++r) {
          double t = 0;
          for (uint64_t k = 0; k < R; ++k) t += M[i * R + k] * Vinv[k * R + r];
          A[i * R + r] = t;
        }
      orc_normalize(A, I, R, lambda, it == 0 ? 2 : 0);
      orc_ata(A, I, R, G[m]);
    }
    /* p_kruskal_norm */
    double norm = 0;
    for (uint64_t a = 0; a < R; ++a)
      for (uint64_t b = 0; b < R; ++b) {
        double h = 1.0;
        for (int m = 0; m < N; ++m) h *= G[m][a * R + b];
        norm += h * lambda[a] * lambda[b];
      }
    norm = fabs(norm);
    /* p_tt_kruskal_inner: M holds the last mode's MTTKRP */
    double inner = 0;
    {
      uint64_t const I = dims[N - 1];
      const double *A = mats[N - 1];
      for (uint64_t r = 0; r < R; ++r) {
        double acc = 0;
        for (uint64_t i = 0; i < I; ++i) acc += A[i * R + r] * M[i * R + r];
        inner += acc * lambda[r];
      }
    }
    double const residual = sqrt(ttnormsq + norm - 2 * inner);
    fit = 1 - residual / sqrt(ttnormsq);
    if (fit_trace) fit_trace[it] = fit;
    if (it > 0 && fabs(fit - oldfit) < tol) {
      ++it;
      break;
    }
    oldfit = fit;
  }
  if (iters_done) *iters_done = it;
  /* cpd_post_process */
  double *tmp = ORC_ALLOC(double, R);
  for (int m = 0; m < N; ++m) {
    orc_normalize(mats[m], dims[m], R, tmp, 2);
    for (uint64_t r = 0; r < R; ++r) lambda[r] *= tmp[r];
  }
  free(tmp);
  for (int m = 0; m < N; ++m) free(G[m]);
  free(Vinv);
  free(M);
  return fit;
}

/* CP-ALS on the memoized model md, or with md == NULL on plain_csfs[m], a
 * tree rooted at mode m (SPLATT_CSF_ALLMODE). See orc_als_core. */
double orc_cpd_als(orc_model *md, const orc_csf *const *plain_csfs,
                   uint64_t nfactors, double *const *mats, double *lambda,
                   uint64_t niters, double tol, double *fit_trace,
                   uint64_t *iters_done) {
  orc_csf const *c0 = md ? md->csf[0] : plain_csfs[0];
  double ttnormsq = 0;
  for (uint64_t n = 0; n < c0->nnz; ++n) ttnormsq += c0->vals[n] * c0->vals[n];
  orc_plain_ctx pc = {plain_csfs, nfactors};
  return orc_als_core(c0->nmodes, c0->dims, ttnormsq, nfactors,
                      md ? orc_mttkrp_model_cb : orc_mttkrp_plain_cb,
                      md ? (void *)md : (void *)&pc, mats, lambda, niters, tol,
                      fit_trace, iters_done);
}

/* ------------------------------------------------------------------------ */
/* Seeded synthetic tensors and an FP64 path for large cases                */
/* ------------------------------------------------------------------------ */

/* Seeded draws with the shapes the benchmark configurations name, the same
 * numbers the library's device generator produces: coordinate m of draw i
 * comes from u = mix64(key_m + i) >> 11 scaled by 2^-53, key_m =
 * mix64(seed * 0x100000001B3 + 0x1000 + m); uniform indices are
 * floor(u * dim), Zipf(alpha) indices the smallest k with u < CDF(k) for
 * P(k) proportional to (k+1)^-alpha; values are u01 of key_N (uniform) or
 * exp(mu + sigma * z) with the Box-Muller z of keys N and N+1 (lognormal).
 * Duplicates are kept (orc_coo_clean sums them). inds is mode-major
 * (nmodes x nnz). Indices and uniform values are bit-identical to the device
 * generator's; lognormal values agree to within a few ulps (the device's
 * cos(pi x), exp and log round differently from glibc's). */
void orc_generate(int nmodes, const uint64_t *dims, uint64_t nnz, const double *alpha,
                  int value_kind, double mu, double sigma, uint64_t seed, uint64_t *inds,
                  double *vals) {
  uint64_t key[ORC_MAXN + 2];
  double *cdf[ORC_MAXN];
  for (int m = 0; m < nmodes + 2; ++m) key[m] = orc_mix64(seed * 0x100000001B3ull + 0x1000u + (uint64_t)m);
  for (int m = 0; m < nmodes; ++m) {
    cdf[m] = NULL;
    if (alpha && alpha[m] > 0) {
      cdf[m] = ORC_ALLOC(double, dims[m]);
      double acc = 0;
      for (uint64_t k = 0; k < dims[m]; ++k) {
        acc += pow((double)(k + 1), -alpha[m]);
        cdf[m][k] = acc;
      }
      for (uint64_t k = 0; k < dims[m]; ++k) cdf[m][k] /= acc;
      cdf[m][dims[m] - 1] = 1.0;
    }
  }
  const double scale = 1.0 / 9007199254740992.0;
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < (int64_t)nnz; ++ii) {
    uint64_t const i = (uint64_t)ii;
    for (int m = 0; m < nmodes; ++m) {
      double const u = (double)(orc_mix64(key[m] + i) >> 11) * scale;
      uint64_t k;
      if (cdf[m] == NULL) {
        k = (uint64_t)(u * (double)dims[m]);
        if (k >= dims[m]) k = dims[m] - 1;
      } else {
        uint64_t lo = 0, hi = dims[m] - 1;
        while (lo < hi) {
          uint64_t const mid = (lo + hi) >> 1;
          if (u < cdf[m][mid])
            hi = mid;
          else
            lo = mid + 1;
        }
        k = lo;
      }
      inds[(uint64_t)m * nnz + i] = k;
    }
    double const u1 = (double)(orc_mix64(key[nmodes] + i) >> 11) * scale;
    if (value_kind == 0) {
      vals[i] = u1;
    } else {
      double const u2 = (double)(orc_mix64(key[nmodes + 1] + i) >> 11) * scale;
      double const z = sqrt(-2.0 * log(1.0 - u1)) * cos(2.0 * M_PI * u2);
      vals[i] = exp(mu + sigma * z);
    }
  }
  for (int m = 0; m < nmodes; ++m) free(cdf[m]);
}

/* MTTKRP of `mode` straight from the coordinates:
 * out[i_mode(n)] += v_n * prod_{m != mode} U_m[i_m(n)], the quantity every
 * CSF kernel of the reference computes (mttkrp.c:241-1682) summed in another
 * order. OpenMP threads take static contiguous ranges of nonzeros into
 * private rows, summed in thread order afterwards, so a run repeats bit for
 * bit at a fixed thread count. */
void orc_mttkrp_coo(int nmodes, uint64_t nnz, const uint64_t *dims, const uint64_t *inds,
                    const double *vals, double *const *mats, uint64_t mode, uint64_t R,
                    double *out) {
  uint64_t const I = dims[mode];
  memset(out, 0, I * R * sizeof(double));
  int nt = 1;
#ifdef _OPENMP
  nt = omp_get_max_threads();
#endif
  double *priv = ORC_ALLOC(double, (uint64_t)nt * I * R);
#pragma omp parallel num_threads(nt)
  {
    int t = 0;
#ifdef _OPENMP
    t = omp_get_thread_num();
#endif
    double *o = priv + (uint64_t)t * I * R;
    double *row = ORC_ALLOC(double, R);
    uint64_t const lo = nnz * (uint64_t)t / (uint64_t)nt, hi = nnz * (uint64_t)(t + 1) / (uint64_t)nt;
    for (uint64_t n = lo; n < hi; ++n) {
      for (uint64_t r = 0; r < R; ++r) row[r] = vals[n];
      for (int m = 0; m < nmodes; ++m) {
        if ((uint64_t)m == mode) continue;
        const double *U = mats[m] + inds[(uint64_t)m * nnz + n] * R;
        for (uint64_t r = 0; r < R; ++r) row[r] *= U[r];
      }
      double *dst = o + inds[mode * nnz + n] * R;
      for (uint64_t r = 0; r < R; ++r) dst[r] += row[r];
    }
    free(row);
  }
#pragma omp parallel for schedule(static)
  for (int64_t x = 0; x < (int64_t)(I * R); ++x) {
    double s = 0;
    for (int t = 0; t < nt; ++t) s += priv[(uint64_t)t * I * R + (uint64_t)x];
    out[x] = s;
  }
  free(priv);
}

typedef struct orc_coo_ctx {
  int nmodes;
  uint64_t nnz, R;
  const uint64_t *dims, *inds;
  const double *vals;
} orc_coo_ctx;

static void orc_mttkrp_coo_cb(void *ctx, double *const *mats, uint64_t mode, double *out) {
  orc_coo_ctx const *c = (orc_coo_ctx const *)ctx;
  orc_mttkrp_coo(c->nmodes, c->nnz, c->dims, c->inds, c->vals, mats, mode, c->R, out);
}

/* CP-ALS (orc_als_core) with the COO MTTKRP: the FP64 reference run for
 * tensors too large for the single-threaded tree restatement. */
double orc_cpd_als_coo(int nmodes, uint64_t nnz, const uint64_t *dims, const uint64_t *inds,
                       const double *vals, uint64_t nfactors, double *const *mats,
                       double *lambda, uint64_t niters, double tol, double *fit_trace,
                       uint64_t *iters_done) {
  double ttnormsq = 0;
  for (uint64_t n = 0; n < nnz; ++n) ttnormsq += vals[n] * vals[n];
  orc_coo_ctx c = {nmodes, nnz, nfactors, dims, inds, vals};
  return orc_als_core(nmodes, dims, ttnormsq, nfactors, orc_mttkrp_coo_cb, &c, mats, lambda,
                      niters, tol, fit_trace, iters_done);
}

int orc_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}
