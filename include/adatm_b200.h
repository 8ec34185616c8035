/*
 * adatm_b200.h -- AdaTM's own entry points (the memoized MTTKRP sequence,
 * its planner and the adaptive CP-ALS) plus the B200 device-resident API.
 *
 * Part 1 keeps the names and argument meaning of the reference's internal
 * headers (src/adatm_rcsf.h, src/adatm_bench.h, src/mttkrp.h,
 * src/adatm_cpd.h), which the reference's CLI and bench call; the SPLATT
 * internal types they take (sptensor_t, matrix_t, thd_info, rank_info,
 * bench_opts) are declared here with the fields those entry points read.
 * Thread scratch (thd_info) and MPI rank info are accepted and ignored.
 *
 * Part 2 is the device-resident interface the B200 build adds: a tensor and
 * an engine (plan, trees, memo rows, factors) stay in HBM across calls, so
 * benchmarks and services avoid host copies per MTTKRP.
 *
 * Every function returns SPLATT_SUCCESS (1) on success and a
 * splatt_error_type, or ADATM_ERROR_CUDA for a CUDA runtime failure, with a
 * message available from adatm_last_error().
 */
#ifndef ADATM_B200_H
#define ADATM_B200_H

#include <stddef.h>
#include <stdint.h>

#include "splatt.h"

#ifdef __cplusplus
extern "C" {
#endif

#define ADATM_ERROR_CUDA 4

/* ======================================================================== */
/* Part 1: SPLATT internal types and the reference's AdaTM entry points     */
/* ======================================================================== */

typedef splatt_idx_t idx_t;
typedef splatt_val_t val_t;

typedef struct {
  idx_t nnz;
  idx_t nmodes;
  idx_t *dims;
  idx_t **ind;
  val_t *vals;
  int tiled;
  int type;
} sptensor_t;

typedef struct {
  idx_t I;
  idx_t J;
  val_t *vals;
  int rowmajor;
} matrix_t;

typedef struct thd_info thd_info;   /* unused by the GPU path; pass NULL */
typedef struct { int rank; } rank_info;

typedef struct {
  idx_t niters;
  idx_t *threads;
  idx_t nruns;
  int write;
  int tile;
  void *perm;
} bench_opts;

/* decide_product_order (reference src/adatm_bench.h:33): product_order[m] has
 * 2*N entries, 1 where MTTKRP m reads factor k unchanged (k < N) or updated
 * (N + k). */
void decide_product_order(sptensor_t *const tt, idx_t **product_order);

/* decide_parameters_auto (reference src/adatm_bench.h:46-51): candidate
 * plans, fiber counts on the GPU, SLIMIT filter, strategy 1 = fewest
 * predicted products, 2 = least predicted space. Returns n_grp; *grp_prop is
 * malloc'd (free o_opt of every group, then the array). */
idx_t decide_parameters_auto(sptensor_t *const tt, idx_t const nfactors, int strategy,
                             idx_t const **product_order, group_properties **grp_prop);

/* decide_candidate_configs / predict_candidates_adaptive /
 * limit_candidates_by_space / choose_candidates_by_strategy (reference
 * src/adatm_bench.h:59-110). */
idx_t decide_candidate_configs(sptensor_t *const tt, idx_t const **product_order,
                               configurations_adaptive **configs);
void predict_candidates_adaptive(sptensor_t *const tt, idx_t const nfactors,
                                 configurations_adaptive *configs, idx_t const nconfigs);
idx_t limit_candidates_by_space(configurations_adaptive const *const configs,
                                idx_t const nconfigs, idx_t **const real_config_locs);
idx_t choose_candidates_by_strategy(configurations_adaptive const *const configs,
                                    idx_t const nconfigs, idx_t const *const real_config_locs,
                                    idx_t const n_real_configs, int strategy);

/* csf_alloc_adaptive (reference src/adatm_rcsf.h:18-23): one tree per
 * group, built on the GPU; the returned host arrays follow the reference
 * layout and the device copies stay resident until splatt_free_csf. */
splatt_csf *csf_alloc_adaptive(sptensor_t *const tt, group_properties *const grp_prop,
                               idx_t const n_grp, double const *const opts, idx_t *n_csf);

/* rcsf_alloc_adaptive (reference src/adatm_rcsf.h:142-149): memo trees that
 * alias the CSF fptr/fids arrays and own nfibs*nfactors values each. Their
 * device rows live in HBM; adatm_rcsf_pull copies them into the host vals. */
rcsf_seq_adaptive *rcsf_alloc_adaptive(splatt_csf *const ct, idx_t const nfactors,
                                       group_properties *const grp_prop, idx_t const n_grp,
                                       idx_t const n_csf, double const *const opts,
                                       idx_t *n_rcsf);

size_t csf_storage_adaptive(splatt_csf const *const tensors, idx_t const n_csf,
                            group_properties *const grp_prop, int const n_grp);
size_t rcsf_storage_adaptive(rcsf_seq_adaptive const *const seq_rcsf, idx_t const n_csf);

/* decide_use_csfs (reference src/mttkrp.h:42-48): tag 0 memo root, 1 memo
 * reuse, 2 recompute. */
void decide_use_csfs(idx_t const nmodes, group_properties *const grp_prop, int const n_grp,
                     idx_t const n_csf, idx_t *use_csfs, idx_t *use_tags);

/* mttkrp_csf_adaptive (reference src/mttkrp.h:51-62): MTTKRP of `mode` into
 * mats[SPLATT_MAX_NMODES] (host, dims[mode] x J), reading mats[0..N-1]. */
void mttkrp_csf_adaptive(splatt_csf const *const tensors, rcsf_seq_adaptive const *const rs_seq,
                         idx_t const n_csf, matrix_t **mats, idx_t const mode,
                         thd_info *const thds, group_properties *const grp_prop,
                         int const n_grp, idx_t const use_csf, idx_t const use_tag,
                         double const *const opts);

/* splatt_cpd_als_adaptive (reference src/adatm_cpd.c:205-215) and
 * cpd_als_iterate_adaptive (reference src/adatm_cpd.h:29-41). */
int splatt_cpd_als_adaptive(splatt_csf const *const tensors, rcsf_seq_adaptive *const rs_seq,
                            splatt_idx_t const n_csf, group_properties const *const grp_prop,
                            splatt_idx_t const n_grp, splatt_idx_t const *const use_csfs,
                            splatt_idx_t const *const use_tags, splatt_idx_t const nfactors,
                            double const *const options, splatt_kruskal *factored);
double cpd_als_iterate_adaptive(splatt_csf const *const tensors, rcsf_seq_adaptive *const rs_seq,
                                splatt_idx_t const n_csf, group_properties const *const grp_prop,
                                splatt_idx_t const n_grp, splatt_idx_t const *const use_csfs,
                                splatt_idx_t const *const use_tags, matrix_t **mats,
                                val_t *const lambda, idx_t const nfactors,
                                rank_info *const rinfo, double const *const opts);

/* bench_adaptm (reference src/adatm_bench.h:22-25): plan, build, then time
 * opts->niters MTTKRP sequences and print per-mode seconds. */
void bench_adaptm(sptensor_t *const tt, matrix_t **mats, bench_opts const *const opts);

/* The reference's report lines, same text: stats_csf_adaptive prints every
 * tree's order, nnz, dims, level order and tiles (adatm_stats.c:19-67),
 * stats_rcsf_adaptive every memo tree of every sequence
 * (adatm_stats.c:70-87), print_group_properties a group list
 * (adatm_debug.c:58-72), iprint_array an index array (adatm_debug.c:5-15).
 * Host only: they read the host views of the trees. */
void stats_csf_adaptive(splatt_csf const *const ct, idx_t const n_csf);
void stats_rcsf_adaptive(rcsf_seq_adaptive const *const seq_rcsfs, idx_t const n_rcsf);
void print_group_properties(group_properties *const grp_prop, idx_t const size, idx_t const nmodes,
                            char *const name);
void iprint_array(idx_t const *const array, idx_t const len, char const *const name);

/* Copy the device memo rows of rs_seq (all sequences, all trees) into their
 * host vals arrays. Not in the reference, whose memo rows live on the host. */
int adatm_rcsf_pull(rcsf_seq_adaptive *rs_seq, idx_t n_rcsf);

/* Number of trees in a splatt_csf array returned by this library (for
 * CSF_ALLOC values whose count the caller cannot infer). */
int adatm_csf_tree_count(splatt_csf const *tensors, int *n);

/* Free a group_properties array returned by decide_parameters_auto. */
void adatm_free_groups(group_properties *grp_prop, idx_t n_grp);

/* ======================================================================== */
/* Part 2: device-resident B200 interface                                   */
/* ======================================================================== */

typedef struct adatm_tensor adatm_tensor;
typedef struct adatm_engine adatm_engine;

/* A memoization plan in flat form. */
typedef struct adatm_plan {
  int nmodes;
  int n_grp;
  uint64_t memo_mode[8];
  uint64_t begin_imten[8];
  uint64_t n_imten[8];
  uint64_t o_opt[8][8];
  uint64_t use_csfs[8];
  uint64_t use_tags[8];
  int space_efficient; /* trees only for memoizing groups (SPLATT_ADAPTIVE_SPACE_EFFICIENT) */
} adatm_plan;

typedef struct adatm_candidate {
  adatm_plan plan;
  uint64_t pspace;
  uint64_t pops;
} adatm_candidate;

/* Message of the calling thread's last library call: empty after a call that
 * succeeded, so the reference's void entry points (mttkrp_csf_adaptive,
 * bench_adaptm) report failures here too; cpd_als_iterate_adaptive returns
 * NaN on failure. */
const char *adatm_last_error(void);

/* Select the CUDA device for the calling thread (the library carries its own
 * CUDA runtime, so a framework's device selection does not reach it). */
int adatm_set_device(int device);

/* COO tensor into HBM. With clean != 0, duplicates are summed in input order
 * and empty slices of every mode are compacted (dims shrink accordingly). */
int adatm_tensor_from_coo(int nmodes, uint64_t nnz, const uint64_t *dims,
                          const uint64_t *const *inds, const double *vals, int clean,
                          adatm_tensor **out);
/* Seeded synthetic tensor, generated and cleaned on the GPU: mode m's
 * indices are uniform (alpha[m] <= 0) or Zipf(alpha[m]) with P(k) ~ (k+1)^-a;
 * values uniform(0,1) (value_kind 0) or lognormal(mu, sigma) (value_kind 1). */
int adatm_tensor_generate(int nmodes, const uint64_t *dims, uint64_t nnz, const double *alpha,
                          int value_kind, double mu, double sigma, uint64_t seed,
                          adatm_tensor **out);
int adatm_tensor_info(const adatm_tensor *t, int *nmodes, uint64_t *nnz, uint64_t *dims);
/* inds: nmodes x nnz (mode-major), vals: nnz */
int adatm_tensor_download(const adatm_tensor *t, uint64_t *inds, double *vals);
void adatm_tensor_free(adatm_tensor *t);

/* Fiber counts per level of the tree in level order `perm` (count_nfibs). */
int adatm_tensor_count_nfibs(const adatm_tensor *t, const uint64_t *perm, uint64_t *nfibs);

/* Analytic plan (decide_parameters_auto); cands (may be NULL) receives up to
 * max_cands candidates with their predictions, *ncands their number, *chosen
 * the reference's returned position. */
int adatm_plan_analytic(const adatm_tensor *t, uint64_t rank, int strategy, adatm_plan *out,
                        adatm_candidate *cands, int max_cands, int *ncands, int *chosen);
/* SPLATT's plain allocations (csf_alloc = SPLATT_CSF_ONEMODE/TWOMODE/ALLMODE). */
int adatm_plan_splatt(const adatm_tensor *t, int csf_alloc, adatm_plan *out);

/* Engine: trees, memo rows and factors for one plan and rank.
 * factor_bf16 != 0 keeps a BF16 copy of every factor for the gathers
 * (accumulation stays FP32). chunk_leaf/chunk_rows: source units per chunk
 * (0 = defaults). The engine copies what it needs from the tensor. */
int adatm_engine_create(const adatm_tensor *t, uint64_t rank, const adatm_plan *plan,
                        int factor_bf16, uint32_t chunk_leaf, uint32_t chunk_rows,
                        adatm_engine **out);
void adatm_engine_free(adatm_engine *e);
int adatm_engine_csf_count(const adatm_engine *e, int *n_csf);
int adatm_engine_csf_shape(const adatm_engine *e, int g, uint64_t *nfibs, uint64_t *dim_perm);
/* Host copies of tree g in the reference layout: fptr[l] (nfibs[l]+1),
 * fids[l] (nfibs[l], fids[0] = root ids), vals (nnz, FP64). */
int adatm_engine_csf_arrays(const adatm_engine *e, int g, uint64_t *const *fptr,
                            uint64_t *const *fids, double *vals);
int adatm_engine_memory(const adatm_engine *e, uint64_t *csf_bytes, uint64_t *memo_bytes);

int adatm_engine_init_factors(adatm_engine *e, uint64_t seed);
int adatm_engine_set_factors(adatm_engine *e, const double *const *mats);
int adatm_engine_get_factors(adatm_engine *e, double *const *mats, double *lambda);

/* MTTKRP of `mode` by the plan (memo root / reuse / recompute) or directly on
 * the mode's tree without memo rows; out: dims[mode] x rank, host FP64. */
int adatm_engine_mttkrp(adatm_engine *e, uint64_t mode, double *out);
int adatm_engine_mttkrp_direct(adatm_engine *e, uint64_t mode, double *out);
/* Memo rows of group g, tree deg, as host FP64 (nfibs[level] x rank). */
int adatm_engine_memo(adatm_engine *e, int g, int deg, double *out);

/* CP-ALS: Grams and ||X||^2, then up to niters sweeps, stopping when
 * |fit - previous| < tol after the first; use_graph captures one sweep in a
 * CUDA graph. trace (may be NULL) receives one fit per sweep. */
int adatm_engine_als(adatm_engine *e, uint64_t niters, double tol, int use_graph, double *fit,
                     uint64_t *iters, double *trace);
int adatm_engine_als_begin(adatm_engine *e, int use_graph);
/* Time `count` sweeps (or MTTKRPs of `mode`, with the row type the sweep
 * uses for that mode) on the engine's stream with CUDA events; *ms is the
 * total. */
int adatm_engine_time_sweeps(adatm_engine *e, int count, float *ms);
int adatm_engine_time_mttkrp(adatm_engine *e, uint64_t mode, int count, float *ms);
int adatm_engine_fit(adatm_engine *e, double *fit);

/* One shard of a tensor split across ranks by root slices (each rank holds
 * an engine on its nonzeros, same dims and plan; factors are replicated).
 * A sweep runs mode by mode: adatm_engine_mttkrp_into writes this shard's
 * MTTKRP of `mode` to a device buffer (dims[mode] x ldr doubles, ldr = R
 * rounded up to 4); the caller sums the ranks' buffers (an all-reduce);
 * adatm_engine_update_from runs the mode's update from the summed buffer;
 * after the last mode adatm_engine_fit_step gives the fit. ||X||^2 is the
 * sum of the shards' adatm_engine_ttnorm values, set on every rank with
 * adatm_engine_set_ttnorm. Calls return when their work is done. Start with
 * adatm_engine_als_begin(e, 0). The reference's only collective is the fit's
 * MPI all-reduce (adatm_cpd.c:147-157); this split adds the MTTKRP sum. */
int adatm_engine_mttkrp_into(adatm_engine *e, uint64_t mode, double *dev_out);
int adatm_engine_update_from(adatm_engine *e, uint64_t mode, const double *dev_M);
int adatm_engine_fit_step(adatm_engine *e, double *fit);
int adatm_engine_ttnorm(adatm_engine *e, double *local);
int adatm_engine_set_ttnorm(adatm_engine *e, double global);
/* Compulsory HBM bytes of the MTTKRP of `mode` as a sweep runs it. With BF16
 * rows, the tree that feeds the last mode (whose MTTKRP gives the fit's
 * inner product) still reads FP32 rows. */
int adatm_engine_mttkrp_bytes(adatm_engine *e, uint64_t mode, double *bytes);
/* Output rows that the mode's MTTKRP walk sums per block in shared memory
 * before adding them to the output (rows hit by very many units of a scatter
 * walk; 0 for contraction walks and unskewed outputs). Diagnostic; no
 * reference counterpart. */
int adatm_engine_hot_rows(adatm_engine *e, uint64_t mode, int *nhot);
/* ------------------------------------------------------------------------ */
/* Batched sweeps of many tensors and the chunk autotuner                   */
/* ------------------------------------------------------------------------ */

/* Time a captured sweep with each (chunk_leaf[i], chunk_rows[i]) and keep the
 * fastest (*best = its index). Runs sweeps: initialise the factors after. */
int adatm_engine_autotune(adatm_engine *e, const uint32_t *chunk_leaf, const uint32_t *chunk_rows,
                          int n, int sweeps, int *best);

/* Contraction walks as a resident grid whose warps claim chunks from a
 * counter (on: the default, fastest for one tensor on the device) or one
 * chunk per warp (off: what a batch uses, so the blocks of walks on
 * concurrent streams interleave). Results agree up to FP32 summation order.
 * Drops a captured sweep. No reference counterpart (a launch-shape control). */
int adatm_engine_set_resident_grid(adatm_engine *e, int on);

/* Walkers per warp in the contraction walks' source loop: 1, 2 or 4 (0 =
 * the default for the rank). With W walkers one warp instruction advances W
 * source units (32/W lanes and up to 4 columns per lane each); refused with
 * SPLATT_ERROR_BADINPUT where W walkers cannot cover the rank. Results agree
 * up to FP32 summation order. Drops a captured sweep. No reference
 * counterpart (a launch-shape control). */
int adatm_engine_set_walkers(adatm_engine *e, int walkers);

/* Unstored tree levels folded into the contraction walks' source loop: 0, 1
 * or 2 (-1, the default: level S-1 whenever it can be, level S-2 too where
 * its nodes hold at most 4 source units on average). A folded level's nodes
 * are not formed: each source unit is multiplied by its ancestors' factor
 * rows directly. Refused with SPLATT_ERROR_BADINPUT outside -1..2. Results
 * agree up to FP32 summation order. Drops a captured sweep. No reference
 * counterpart (a kernel-shape control). */
int adatm_engine_set_fold(adatm_engine *e, int fold);

/* Deterministic accumulation, on by default (on != 0): no float atomics
 * anywhere in the MTTKRPs. Contractions write the partial sums of the tree
 * nodes that chunk boundaries cut to per-chunk rows and sum them per node in
 * chunk order (always, in both settings); scatters, and contractions whose
 * output level is below the root, visit every output row's contributions in
 * a stable order by row. Output rows are FP64 sums. Sweeps then repeat bit
 * for bit from the same start, on one device and build. Costs extra device
 * memory (per-chunk rows, sorted unit lists, prefix rows). Off (on == 0),
 * scatters add into the FP64 output rows with atomics (order-dependent in
 * the last bits). Drops a captured sweep. No reference counterpart: the
 * reference's locked OpenMP scatters (mttkrp.c:13-14,121-125) sum in thread
 * order. */
int adatm_engine_set_deterministic(adatm_engine *e, int on);

/* One ALS iteration of every engine in one CUDA graph (each engine on its
 * own branch). The engines must outlive the batch. */
typedef struct adatm_batch adatm_batch;
int adatm_batch_create(adatm_engine *const *engines, int n, adatm_batch **out);
/* Grams and norms of every engine, then the graph capture. */
int adatm_batch_begin(adatm_batch *b);
/* `count` graph launches timed with CUDA events (*ms total). */
int adatm_batch_time_sweeps(adatm_batch *b, int count, float *ms);
int adatm_batch_kernels(const adatm_batch *b, int *per_sweep);
void adatm_batch_free(adatm_batch *b);

/* ------------------------------------------------------------------------ */
/* Learned plan model (replaces the analytic cost model of                  */
/* decide_parameters_auto, reference src/adatm_bench.c:145-272, which stays  */
/* the fallback).                                                            */
/* ------------------------------------------------------------------------ */

#define ADATM_PLAN_FEATURES 16

/* Candidate plans of decide_candidate_configs for the tensor, with
 * ADATM_PLAN_FEATURES features per candidate (row-major into `features`,
 * room for max_cands rows) and each candidate's exact device bytes. */
int adatm_plan_features(const adatm_tensor *t, uint64_t rank, float *features, double *bytes,
                        adatm_candidate *cands, int max_cands, int *ncands);

/* A fully connected network: widths[0] inputs, ReLU hidden layers
 * widths[1..nwidths-2], one linear output; He-uniform weights from seed. */
typedef struct adatm_mlp adatm_mlp;
int adatm_mlp_create(int nwidths, const int *widths, uint64_t seed, adatm_mlp **out);
void adatm_mlp_free(adatm_mlp *m);
/* Parameters, layer by layer: W (out x in, row-major) then b (out). */
int adatm_mlp_nparams(const adatm_mlp *m, uint64_t *n);
int adatm_mlp_set_params(adatm_mlp *m, const float *params);
int adatm_mlp_get_params(const adatm_mlp *m, float *params);
/* Y[rows] = net(X[rows x widths[0]]) on the GPU (host buffers). */
int adatm_mlp_forward(adatm_mlp *m, const float *X, uint64_t rows, float *Y);
/* Mean squared error against T and its gradient (nparams floats, the
 * parameter layout), by the GPU backward kernels. */
int adatm_mlp_gradient(adatm_mlp *m, const float *X, const float *T, uint64_t rows, float *grad,
                       double *loss);
/* Adam on seeded minibatches on the GPU; *loss = mean loss of the last epoch. */
int adatm_mlp_train(adatm_mlp *m, const float *X, const float *T, uint64_t rows, int epochs,
                    int batch, float lr, uint64_t seed, double *loss);

/* The learned plan: every candidate's features, standardised by feat_mean /
 * feat_std, are scored by the network (predicted log sweep time) and the
 * lowest-scoring candidate within the reference's storage limit is chosen.
 * With m == NULL, or a non-finite score, the analytic plan is returned and
 * *used_model = 0. */
int adatm_plan_learned(const adatm_tensor *t, uint64_t rank, adatm_mlp *m, const float *feat_mean,
                       const float *feat_std, adatm_plan *out, int *chosen, int *used_model);

/* G = A^T A in FP64 (R x R, row-major, device) of the device row matrix A
 * (rows x ldr floats, 16-byte aligned, first R <= 128 columns used, ldr a
 * multiple of 4): the Gram step of the CP-ALS update, with its per-block
 * partial sums in workspace the call allocates and frees. Synchronous. */
int adatm_gram(const float *A, uint64_t rows, int R, int ldr, double *G);

/* adatm_gram without any device allocation; no counterpart in the reference.
 * For callers that cannot allocate device memory at the call (a caching
 * allocator already holds the free HBM, or cudaFree's device-wide
 * synchronisation is not acceptable): the partial sums live in a fixed
 * 2 MiB device array, so R must be <= 64 (SPLATT_ERROR_BADINPUT otherwise).
 * Runs on `stream` (a cudaStream_t; NULL = the legacy default stream) and
 * returns after it completes. Calls that overlap in time on one device race
 * on the shared array. The first call on a device resolves the array's
 * address; make it once before any stream capture. After cudaDeviceReset
 * the resolved address is stale: do not call it again in that process. */
int adatm_gram_noalloc(const float *A, uint64_t rows, int R, int ldr, double *G, void *stream);

/* Number of kernel launches of one sweep and of one MTTKRP of `mode`. */
int adatm_engine_launch_counts(adatm_engine *e, uint64_t mode, int *per_sweep, int *per_mttkrp);

#ifdef __cplusplus
}
#endif

#endif
