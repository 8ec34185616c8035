/*
 * adatm_oracle.h -- CPU FP64 oracle for the AdaTM memoized MTTKRP sequence
 * and the CP-ALS sweep around it.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker: tests/, the smoke check and
 * bench.py's cpu_baseline leg call it to validate and to time the reference
 * algorithm on host cores. The product library never links or calls it.
 *
 * Every function restates the reference algorithm (hpcgarage/AdaTM, a patch
 * over SPLATT v1.1.1) from its source; each definition in adatm_oracle.c
 * cites the reference file:line it follows. Types follow the reference
 * defaults: 64-bit indices, double values (include/splatt.h:26-31).
 */
#ifndef ADATM_ORACLE_H
#define ADATM_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#define ORC_MAXN 16

/* CSF tree in the reference layout (include/splatt.h:235-287, one tile). */
typedef struct orc_csf {
  int nmodes;
  uint64_t nnz;
  uint64_t dims[ORC_MAXN];
  uint64_t dim_perm[ORC_MAXN];
  uint64_t nfibs[ORC_MAXN];
  uint64_t *fptr[ORC_MAXN]; /* fptr[l] for l <= N-2, length nfibs[l]+1 */
  uint64_t *fids[ORC_MAXN]; /* fids[0] == NULL (untiled), fids[l] for l >= 1 */
  uint64_t *root_ids;       /* index of each root slice (kept beside the
                               reference layout; equals s after compaction) */
  double *vals;
} orc_csf;

/* One MTTKRP group (include/splatt.h:302-318). */
typedef struct orc_grp {
  uint64_t memo_mode;
  uint64_t begin_imten;
  uint64_t n_imten;
  uint64_t o_opt[ORC_MAXN];
} orc_grp;

/* One candidate configuration (include/splatt.h:323-336). */
typedef struct orc_config {
  uint64_t n_grp;
  orc_grp grp[ORC_MAXN];
  uint64_t pspace;
  uint64_t pops;
} orc_config;

/* The whole memoized model: plan, CSFs, memo trees. */
typedef struct orc_model {
  int nmodes;
  uint64_t nfactors;
  uint64_t dims[ORC_MAXN];
  uint64_t n_grp;
  orc_grp grp[ORC_MAXN];
  uint64_t n_csf;
  orc_csf *csf[ORC_MAXN];
  uint64_t use_csfs[ORC_MAXN];
  uint64_t use_tags[ORC_MAXN];
  double *memo[ORC_MAXN][ORC_MAXN]; /* memo[g][deg]: F_{b-1-deg} x R */
  uint64_t memo_rows[ORC_MAXN][ORC_MAXN];
} orc_model;

/* --- COO helpers ------------------------------------------------------- */
void orc_sort_order(int nmodes, uint64_t nnz, const uint64_t *dims,
                    const uint64_t *inds, const uint64_t *perm,
                    uint64_t *order);
uint64_t orc_coo_clean(int nmodes, uint64_t nnz, uint64_t *dims,
                       uint64_t *inds, double *vals);

/* --- CSF ----------------------------------------------------------------- */
orc_csf *orc_csf_build(int nmodes, uint64_t nnz, const uint64_t *dims,
                       const uint64_t *inds, const double *vals,
                       const uint64_t *dim_perm);
void orc_csf_free(orc_csf *ct);
void orc_count_nfibs(int nmodes, uint64_t nnz, const uint64_t *dims,
                     const uint64_t *inds, const uint64_t *o_opt,
                     uint64_t *nfibs);
void orc_splatt_perm(int nmodes, const uint64_t *dims, int which,
                     uint64_t root, uint64_t *perm);

/* --- planner ------------------------------------------------------------- */
int orc_candidate_configs(int nmodes, const uint64_t *dims,
                          orc_config *configs, int max_configs);
void orc_predict_candidates(int nmodes, uint64_t nnz, const uint64_t *dims,
                            const uint64_t *inds, uint64_t nfactors,
                            orc_config *configs, int nconfigs);
int orc_choose_config(const orc_config *configs, int nconfigs, int strategy,
                      double slimit);
uint64_t orc_plan(int nmodes, uint64_t nnz, const uint64_t *dims,
                  const uint64_t *inds, uint64_t nfactors, int strategy,
                  orc_grp *grp_out, orc_config *all_out, int *nconfigs_out);
void orc_decide_use_csfs(int nmodes, const orc_grp *grp, uint64_t n_grp,
                         uint64_t n_csf, uint64_t *use_csfs,
                         uint64_t *use_tags);
void orc_pair_sort(uint64_t *x, uint64_t *y, uint64_t n);

/* --- model / MTTKRP ------------------------------------------------------- */
orc_model *orc_model_build(int nmodes, uint64_t nnz, const uint64_t *dims,
                           const uint64_t *inds, const double *vals,
                           uint64_t nfactors, uint64_t n_grp,
                           const orc_grp *grp);
void orc_model_free(orc_model *md);
void orc_mttkrp_adaptive(orc_model *md, double *const *mats, uint64_t mode,
                         double *out);
void orc_mttkrp_csf(const orc_csf *ct, double *const *mats, uint64_t mode,
                    uint64_t nfactors, double *out);

/* --- CP-ALS -------------------------------------------------------------- */
void orc_factor_init(uint64_t seed, uint64_t mode, uint64_t rows,
                     uint64_t nfactors, double *out);
double orc_cpd_als(orc_model *md, const orc_csf *const *plain_csfs,
                   uint64_t nfactors, double *const *mats, double *lambda,
                   uint64_t niters, double tol, double *fit_trace,
                   uint64_t *iters_done);


/* --- seeded synthetic tensors; FP64 COO path for large cases ------------- */
void orc_generate(int nmodes, const uint64_t *dims, uint64_t nnz, const double *alpha,
                  int value_kind, double mu, double sigma, uint64_t seed, uint64_t *inds,
                  double *vals);
void orc_mttkrp_coo(int nmodes, uint64_t nnz, const uint64_t *dims, const uint64_t *inds,
                    const double *vals, double *const *mats, uint64_t mode, uint64_t R,
                    double *out);
double orc_cpd_als_coo(int nmodes, uint64_t nnz, const uint64_t *dims, const uint64_t *inds,
                       const double *vals, uint64_t nfactors, double *const *mats,
                       double *lambda, uint64_t niters, double tol, double *fit_trace,
                       uint64_t *iters_done);
/* OpenMP threads of the parallel oracle paths (n > 0 sets them); returns
 * the count in use. */
int orc_threads(int n);

#endif
