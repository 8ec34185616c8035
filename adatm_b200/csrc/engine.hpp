// engine.hpp -- one tensor resident in HBM with its plan, CSF trees, memo
// rows, factor matrices and the CP-ALS sweep.
#pragma once

#include <map>
#include <memory>
#include <tuple>
#include <vector>

#include "als.cuh"
#include "mttkrp.cuh"
#include "planner.hpp"

namespace adatm {

struct EngineOptions {
  FactorType factor_type = FactorType::F32;
  uint32_t chunk_leaf = 256;  // source units per chunk (one warp), nonzero sources
  uint32_t chunk_rows = 128;  // source units per chunk (one warp), memo-row sources
  int max_iters = 1024;       // capacity of the device fit trace
  // contraction walks as a resident grid whose warps claim chunks (fastest
  // for one tensor on the device); off, one chunk per warp, so the blocks of
  // walks running side by side on other streams interleave
  bool resident_grid = true;
  // walkers per warp in the contraction source loop (0 = default_walkers(R))
  int walkers = 0;
  // unstored levels folded into the contraction source loop (0..2; -1 =
  // chosen from each tree's fan-out)
  int fold = -1;
  // no float atomics (the default): every MTTKRP output and memo row is
  // summed in an order fixed by the tree, in FP64 across chunks, so sweeps
  // repeat bit for bit; off, scatters add into the FP64 output rows with
  // atomics
  bool deterministic = true;
};

class Engine {
 public:
  // trees: prebuilt CSF trees of the plan (empty = build them here)
  Engine(std::shared_ptr<const DevCoo> coo, std::vector<std::shared_ptr<DevCsf>> trees,
         uint64_t rank, const Plan &plan, const EngineOptions &opt, cudaStream_t stream);
  ~Engine();
  Engine(const Engine &) = delete;
  Engine &operator=(const Engine &) = delete;

  int nmodes() const { return coo_->nmodes; }
  uint64_t rank() const { return R_; }
  int ldr() const { return ldr_; }
  uint64_t nnz() const { return coo_->nnz; }
  const uint64_t *dims() const { return coo_->dims; }
  const Plan &plan() const { return plan_; }
  const DevCsf &csf(int g) const { return *csf_[g]; }
  int n_csf() const { return (int)csf_.size(); }
  const DevCoo &coo() const { return *coo_; }
  const std::vector<std::shared_ptr<DevCsf>> &trees() const { return csf_; }
  int kernels_per_mttkrp(int mode) const;
  int kernels_per_sweep() const;
  cudaStream_t stream() const { return stream_; }
  FactorType factor_type() const { return opt_.factor_type; }
  const TreeWalk &walk(int mode) const { return *walk_[mode]; }
  size_t memo_bytes() const;
  size_t csf_bytes() const;

  // factors
  void init_factors(uint64_t seed);
  void set_factors(const double *const *host);          // dims[m] x R each
  void get_factors(double *const *host);
  void get_lambda(double *host) const;
  // The factors as the reference returns them after cpd_post_process: every
  // column scaled to unit 2-norm (norms from the device Grams' diagonals,
  // which the sweep keeps current), lambda multiplied by those norms; one
  // pass over the downloaded rows.
  void get_normalized(double *const *host, double *lambda);
  // One sweep whose result comes back as get_normalized's does, but mode by
  // mode: each mode's rows and Gram are copied out as soon as its update
  // ends and normalised on the host while the later modes run. Returns the
  // sweep's fit.
  double sweep_download(double *const *host, double *lambda);
  float *factor(int m) { return A_[m].get(); }

  // MTTKRP of `mode` following the plan (tags 0/1/2) into out (dims x ldr
  // FP64, zeroed here). Memo reuse (tag 1) expects the group's memo root to have
  // run on the current factors of the memoized levels.
  void mttkrp(int mode, double *out);
  // same, with the factor rows read in the given precision
  void mttkrp_as(int mode, double *out, FactorType ft);
  // Row type of mode `mode`'s MTTKRP inside a sweep.
  FactorType sweep_type(int mode) const;
  // MTTKRP of `mode` recomputed on its group's tree without memo rows.
  void mttkrp_direct(int mode, double *out);
  // MTTKRP of `mode` the way a reference caller names it: on tree `tree`
  // with tag 0 (root MTTKRP; it stores the tree's memo rows when its group
  // memoizes), 1 (reuse of the tree's memo rows) or 2 (recompute from the
  // leaves), as mttkrp_csf_adaptive dispatches (mttkrp.c:2037-2090). The
  // walk is built on first use and kept.
  void mttkrp_with(int mode, int tree, int tag, double *out);
  // Whether (mode, tree, tag) is a valid request on this plan's trees:
  // throws BadInput naming the problem (tag 0 on a mode that is not the
  // tree's root, tag 2 on the root, tag 1 on a tree without memo rows or
  // whose memo rows lie above the mode's level).
  void check_use(int mode, int tree, int tag) const;
  // Run the sweep with these per-mode trees and tags (a reference caller's
  // use_csfs / use_tags) instead of the plan's: checked with check_use, and
  // a tag-1 mode needs the root MTTKRP (tag 0) of its tree at an earlier
  // mode of the sweep, which writes the memo rows it reads. Rebuilds the
  // walks and drops a captured sweep when they change.
  void set_use(const uint64_t *use_csfs, const uint64_t *use_tags);
  double *mttkrp_buffer() { return M_.get(); }
  const float *memo_rows(int g, int deg) const { return memo_[g][deg].get(); }

  // One shard of a tensor split across ranks (the nonzeros of some root
  // slices; factors replicated): the sweep runs mode by mode with the sum of
  // the ranks' MTTKRPs taken outside the engine between the two halves.
  //   mttkrp_into(m, buf): this shard's MTTKRP of mode m into a device
  //     buffer (dims[m] x ldr FP64), finished when the call returns;
  //   update_from(m, buf): the mode-m update (Gram inverse, A = M V^-1,
  //     normalisation, Gram, the fit's inner product for the last mode)
  //     from the summed MTTKRP, finished when the call returns;
  //   fit_step(): the fit from the Grams, lambda and the inner product.
  // ttnorm_local() / set_ttnorm(): this shard's ||X||^2 and the global one.
  void mttkrp_into(int mode, double *dev_out);
  void update_from(int mode, const double *dev_M);
  double fit_step();
  double ttnorm_local();
  void set_ttnorm(double v);

  // CP-ALS
  void als_begin();                      // Grams, ||X||^2, iteration counter
  void sweep();                          // one ALS iteration (graph replay if captured)
  void sweep_eager();                    // one ALS iteration, plain launches
  void capture_graph();
  double fit_host();                     // last fit (synchronises)
  int iter_host();
  void fit_trace(double *host, int n);

  // compulsory HBM bytes of the MTTKRP of `mode` (roofline numerator)
  double mttkrp_bytes(int mode) const;

  // Rebuild the walk schedules with other chunk sizes (drops a captured
  // graph). Factors, Grams and memo rows stay as they are.
  void set_chunks(uint32_t chunk_leaf, uint32_t chunk_rows);
  // Contraction grid shape (EngineOptions::resident_grid); drops a captured
  // sweep.
  void set_resident_grid(bool on);
  // Walkers per warp of the contraction walks (1, 2, 4; 0 = the default
  // for the rank); drops a captured sweep.
  void set_walkers(int walkers);
  // Levels folded into the contraction source loop (0, 1, 2; -1 = chosen
  // from the fan-out); drops a captured sweep.
  void set_fold(int fold);
  // Deterministic accumulation on or off (rebuilds the walks, drops a
  // captured sweep; factors, Grams and memo rows stay).
  void set_deterministic(bool on);
  bool deterministic() const { return opt_.deterministic; }
  uint32_t chunk_leaf() const { return opt_.chunk_leaf; }
  uint32_t chunk_rows() const { return opt_.chunk_rows; }
  // Time `count` graph-replayed sweeps (CUDA events, ms total).
  float time_sweeps(int count);
  // Chunk autotuner: time a captured sweep with every (leaf, rows) pair and
  // keep the fastest; returns its index. Runs sweeps, so it changes the
  // factors: initialise them afterwards.
  int autotune(const std::vector<std::pair<uint32_t, uint32_t>> &options, int sweeps);

 private:
  void build_walks();
  std::unique_ptr<TreeWalk> make_walk(int mode, int tree, int tag);
  LevelFactors level_factors(int g, FactorType ft) const;

  std::shared_ptr<const DevCoo> coo_;
  uint64_t R_;
  int ldr_;
  Plan plan_;
  EngineOptions opt_;
  cudaStream_t stream_;
  std::vector<std::shared_ptr<DevCsf>> csf_;
  DevBuf<float> memo_[kMaxModes][kMaxModes];
  std::unique_ptr<TreeWalk> walk_[kMaxModes];
  std::unique_ptr<TreeWalk> direct_[kMaxModes];
  std::map<std::tuple<int, int, int>, std::unique_ptr<TreeWalk>> custom_;  // by (mode, tree, tag)
  DevBuf<float> A_[kMaxModes];
  DevBuf<__nv_bfloat16> Ab_[kMaxModes];
  DevBuf<double> G_[kMaxModes];
  DevBuf<double> M_;
  AlsWork w_;
  bool ttnorm_ready_ = false;    // ||X||^2 computed (the tensor never changes)
  float *staging_ = nullptr;     // pinned host rows for factor transfers
  size_t staging_n_ = 0;
  float *staging(size_t n);
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t graph_exec_ = nullptr;
  void drop_graph();
  // Side stream for the Gram inverse of a mode, which overlaps that mode's
  // MTTKRP (it reads only the other modes' Grams); fork / join events.
  cudaStream_t side_ = nullptr;
  cudaEvent_t fork_ = nullptr, join_ = nullptr;
  cudaEvent_t staged_ = nullptr;  // after the last copy that reads the staging rows
  bool staged_pending_ = false;
  // Downloads that overlap a sweep: each mode's update records updated_[m]
  // (an event node of the captured sweep); the copy stream takes the mode's
  // rows and Gram once it fires and records landed_[m] (landed_[N]: lambda).
  cudaStream_t copy_ = nullptr;
  cudaEvent_t updated_[kMaxModes] = {};
  cudaEvent_t landed_[kMaxModes + 1] = {};
};

// Many independent tensors swept together: one CUDA graph holds one ALS
// iteration of every engine, each engine's kernels on a branch of its own
// (its stream, forked from and joined to the batch's stream), so the small
// launches of uneven tensors overlap on the GPU and the host launches one
// graph per iteration. The engines must outlive the batch.
class BatchSweep {
 public:
  BatchSweep(std::vector<Engine *> engines, cudaStream_t stream);
  ~BatchSweep();
  BatchSweep(const BatchSweep &) = delete;
  BatchSweep &operator=(const BatchSweep &) = delete;
  void begin();                 // als_begin of every engine, then capture
  void sweep();                 // one graph launch
  float time_sweeps(int count); // CUDA events on the batch stream, ms total
  int kernels_per_sweep() const;

 private:
  std::vector<Engine *> e_;
  cudaStream_t s_;
  cudaEvent_t fork_ = nullptr;
  std::vector<cudaEvent_t> join_;
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t exec_ = nullptr;
};

}  // namespace adatm
