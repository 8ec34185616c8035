// planner.hpp -- memoization plans for the MTTKRP sequence.
//
// A plan is the reference's group list (include/splatt.h:302-318): group g
// computes the MTTKRP of memo_mode from scratch on a CSF tree in o_opt order
// and keeps n_imten memo levels for the followers of the group. SPLATT's
// plain allocations (ONEMODE / TWOMODE / ALLMODE) are expressed as plans too,
// so one dispatcher serves every CSF_ALLOC value.
#pragma once

#include <vector>

#include "csf_build.cuh"

namespace adatm {

struct Group {
  uint64_t memo_mode = 0;
  uint64_t begin_imten = 0;
  uint64_t n_imten = 0;
  uint64_t o_opt[kMaxModes] = {0};
};

struct Plan {
  int nmodes = 0;
  int n_grp = 0;
  Group grp[kMaxModes];
  // per mode: which tree and which MTTKRP (0 root, 1 memo reuse, 2 recompute)
  uint64_t use_csfs[kMaxModes] = {0};
  uint64_t use_tags[kMaxModes] = {0};
  int n_csf = 0;
  // tree t is built in the order of group tree_group[t] (identity except in
  // SPACE_EFFICIENT plans, whose trees are the memoizing groups only)
  int tree_group[kMaxModes] = {0, 1, 2, 3, 4, 5, 6, 7};
  bool space_efficient = false;
  const Group &tree(int t) const { return grp[tree_group[t]]; }
};

struct Candidate {
  Plan plan;
  uint64_t pspace = 0;
  uint64_t pops = 0;
};

// decide_product_order + decide_candidate_configs (adatm_bench.c:62-74,
// 276-458).
std::vector<Candidate> candidate_configs(int nmodes, const uint64_t *dims);

// predict_candidates_adaptive (adatm_bench.c:145-272) with the fiber counts
// of every group's tree taken from the GPU construction kernels.
void predict_candidates(const DevCoo &coo, uint64_t nfactors, std::vector<Candidate> &cands,
                        cudaStream_t s);

// limit_candidates_by_space + choose_candidates_by_strategy
// (adatm_bench.c:77-142), returning the position the reference returns.
int choose_candidate(const std::vector<Candidate> &cands, int strategy, double slimit);

// decide_parameters_auto (adatm_bench.c:462-508): the analytic plan.
Plan plan_analytic(const DevCoo &coo, uint64_t nfactors, int strategy,
                   std::vector<Candidate> *all, cudaStream_t s);

// Features of every candidate plan for the learned plan model: tensor shape
// (order, nnz, rank, dims) and, from the exact fiber counts of each group's
// tree (counted on the GPU), the work of the N walks the plan runs -- units
// of contracting and scattering walks, their upper-level items, memo rows
// stored, scatter fan-in per output row -- and its exact storage. Row c of
// `features` (kPlanFeatures floats) belongs to cands[c]; `bytes` receives the
// exact device bytes of each candidate's trees plus memo rows.
constexpr int kPlanFeatures = 16;
void plan_features(const DevCoo &coo, uint64_t nfactors, const std::vector<Candidate> &cands,
                   std::vector<float> &features, std::vector<double> &bytes, cudaStream_t s);

// decide_use_csfs (mttkrp.c:1940-2033); fills plan.use_csfs/use_tags/n_csf.
void decide_use_csfs(Plan &p);
// SPACE_EFFICIENT plans (adatm_rcsf.c:528-552, mttkrp.c:1976-2029): trees
// only for the groups that memoize; every other group's modes recompute
// (tag 2) on the tree locate_ind_special names. A plan with one group, or
// with no memoizing group, stays TIME_EFFICIENT.
void decide_use_csfs_space(Plan &p);

// SPLATT's plain allocations as plans: ONEMODE (one tree, modes by dimension
// ascending), TWOMODE (that tree plus one rooted at the largest mode),
// ALLMODE (one tree rooted at every mode, the others by dimension
// ascending).
Plan plan_splatt(int nmodes, const uint64_t *dims, int csf_alloc);

// SPLATT's dimension orders (see plan_splatt).
void splatt_perm(int nmodes, const uint64_t *dims, bool root_first, uint64_t root, uint64_t *perm);

// The reference's pair_sort (adatm_sort.c:10-75).
void pair_sort(uint64_t *x, uint64_t *y, uint64_t n);

}  // namespace adatm
