// planner.cpp -- the analytic memo planner of the reference, with fiber
// counts from the GPU, plus SPLATT's plain allocations as plans.
#include "planner.hpp"

#include <cmath>
#include <cstring>
#include <map>

namespace adatm {

namespace {

// first index of the smallest entry above `con` (adatm_utils.c:33-51);
// n when none exists
uint64_t argmin_above(const uint64_t *a, uint64_t n, uint64_t con) {
  uint64_t best = n;
  for (uint64_t i = 0; i < n; ++i)
    if (a[i] > con && (best == n || a[i] < a[best])) best = i;
  return best;
}

// smallest entry above `con` (adatm_utils.c:80-97); 0 when none exists
uint64_t min_above(const uint64_t *a, uint64_t n, uint64_t con) {
  uint64_t best = 0;
  bool found = false;
  for (uint64_t i = 0; i < n; ++i)
    if (a[i] > con && (!found || a[i] < best)) {
      best = a[i];
      found = true;
    }
  return best;
}

void pair_sort_part(uint64_t *x, uint64_t *y, uint64_t lo, uint64_t hi) {
  // Same partition steps as the reference so that ties land identically:
  // pivot taken from the middle and parked at `lo`, then a two-cursor sweep.
  uint64_t i = lo + 1, j = hi - 1;
  const uint64_t mid = lo + (hi - lo) / 2;
  const uint64_t px = x[mid], py = y[mid];
  x[mid] = x[lo];
  y[mid] = y[lo];
  while (i < j) {
    if (y[i] > py) {
      if (y[j] < py) {
        std::swap(x[i], x[j]);
        std::swap(y[i], y[j]);
        ++i;
      }
      --j;
    } else {
      if (y[j] > py) --j;
      ++i;
    }
  }
  if (y[i] > py) --i;
  x[lo] = x[i];
  y[lo] = y[i];
  x[i] = px;
  y[i] = py;
  if (i > lo + 1) pair_sort_part(x, y, lo, i);
  if (hi - (i + 1) > 1) pair_sort_part(x, y, i + 1, hi);
}

}  // namespace

void pair_sort(uint64_t *x, uint64_t *y, uint64_t n) {
  if (n > 1) pair_sort_part(x, y, 0, n);
}

std::vector<Candidate> candidate_configs(int nmodes, const uint64_t *dims) {
  const uint64_t N = (uint64_t)nmodes;
  // uses[m][k]: MTTKRP m reads factor k unchanged (k < N) or updated (k >= N)
  uint64_t uses[kMaxModes][2 * kMaxModes] = {{0}};
  for (uint64_t m = 0; m < N; ++m) {
    for (uint64_t i = m + 1; i < N; ++i) uses[m][i] = 1;
    for (uint64_t i = 0; i < m; ++i) uses[m][N + i] = 1;
  }
  std::vector<Candidate> out;
  const uint64_t ncal = (uint64_t)std::ceil((double)N / std::sqrt(2.0 * (double)(N - 1)));
  for (uint64_t ng = 1; ng <= ncal + 1; ++ng) {
    const uint64_t avg = N / ng;
    uint64_t rest = N % ng;
    if (avg == 1 && rest > 0) continue;
    if (ng >= N) continue;
    uint64_t maxn[kMaxModes + 2] = {0}, begin[kMaxModes + 2] = {0}, memo[kMaxModes + 2] = {0};
    uint64_t n_grp = ng;
    if (ng == 1) {
      // one memo group for mode 0 plus a plain tree for mode N-1
      n_grp = 2;
      maxn[0] = N - 2;
      begin[0] = N - 1;
      memo[1] = N - 1;
      begin[1] = 1;
    } else {
      for (uint64_t g = 0; g < ng; ++g) {
        maxn[g] = rest > 0 ? avg : avg - 1;
        if (rest > 0) --rest;
        begin[g] = maxn[g] + 1;
        if (g > 0) memo[g] = memo[g - 1] + maxn[g - 1] + 1;
      }
    }
    const uint64_t variants = min_above(maxn, ncal + 1, 0);
    for (uint64_t v = 0; v < variants; ++v) {
      Candidate c;
      c.plan.nmodes = nmodes;
      c.plan.n_grp = (int)n_grp;
      for (uint64_t g = 0; g < n_grp; ++g) {
        Group &gp = c.plan.grp[g];
        gp.memo_mode = memo[g];
        gp.begin_imten = begin[g];
        gp.n_imten = memo[g] != N - 1 ? maxn[g] - v : 0;
        // o_opt: memo mode, then factors by how often the group's MTTKRPs
        // use them (fewest first), the tail from begin_imten by dimension
        uint64_t total[2 * kMaxModes] = {0}, times[2 * kMaxModes] = {0}, order[kMaxModes] = {0};
        for (uint64_t j = memo[g]; j <= memo[g] + maxn[g]; ++j)
          for (uint64_t k = 0; k < 2 * N; ++k) total[k] += uses[j][k];
        for (uint64_t k = 0; k < 2 * N; ++k) times[k] = uses[memo[g]][k] ? total[k] : 0;
        order[0] = memo[g];
        for (uint64_t j = 1; j < N; ++j) {
          uint64_t k = argmin_above(times, 2 * N, 0);
          times[k] = 0;
          order[j] = k >= N ? k - N : k;
        }
        const uint64_t tail = N - gp.begin_imten;
        uint64_t tx[kMaxModes], ty[kMaxModes];
        for (uint64_t j = 0; j < tail; ++j) {
          tx[j] = order[gp.begin_imten + j];
          ty[j] = dims[tx[j]];
        }
        pair_sort(tx, ty, tail);
        gp.o_opt[0] = memo[g];
        for (uint64_t j = 1; j < gp.begin_imten; ++j) gp.o_opt[j] = order[j];
        for (uint64_t j = 0; j < tail; ++j) gp.o_opt[gp.begin_imten + j] = tx[j];
      }
      out.push_back(c);
    }
  }
  return out;
}

void predict_candidates(const DevCoo &coo, uint64_t R, std::vector<Candidate> &cands,
                        cudaStream_t s) {
  const int N = coo.nmodes;
  const uint64_t nnz = coo.nnz;
  std::map<std::vector<uint64_t>, std::vector<uint64_t>> cache;
  auto counts_for = [&](const Group &g) {
    std::vector<uint64_t> key(g.o_opt, g.o_opt + N);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    std::vector<uint64_t> nf(N, 0);
    csf_count(coo, g.o_opt, nf.data(), s);
    nf[N - 1] = nnz;
    cache[key] = nf;
    return nf;
  };
  auto csf_bytes = [&](const std::vector<uint64_t> &nf) {  // adatm_rcsf.c:329-345
    uint64_t b = nnz * 8 + nnz * 8;
    for (int m = 0; m < N - 1; ++m) b += (nf[m] + 1) * 8 + nf[m] * 8;
    return b;
  };
  auto memo_bytes = [&](const Group &g, const std::vector<uint64_t> &nf) {  // :347-363
    uint64_t b = 0;
    for (uint64_t i = 0; i < g.n_imten; ++i) b += nf[g.begin_imten - i] * R * 8;
    return b;
  };
  auto csf_ops = [&](const std::vector<uint64_t> &nf) {  // :365-379
    uint64_t o = 0;
    for (int m = 0; m < N; ++m) o += nf[m] * R * 2;
    return o;
  };
  auto memo_ops = [&](const Group &g, uint64_t reuse, const std::vector<uint64_t> &nf) {  // :382-406
    if (g.n_imten == 0) return (uint64_t)0;
    uint64_t o = 0;
    const uint64_t end = g.begin_imten - g.n_imten + 1;
    for (uint64_t i = 1; i <= reuse; ++i) {
      if (i < end) o += nf[end - 1] * R * 2;
      else if (i < g.begin_imten) o += nf[i] * R * 2;
    }
    return o;
  };
  // Fiber counts are taken afresh only when the group count changes; a
  // configuration with the same group count as its predecessor evaluates
  // every group with the counts of the last group counted, as the reference
  // does (adatm_bench.c:246-261). This decides the reference's pick.
  std::vector<uint64_t> last;
  uint64_t cbytes = 0, cops = 0, reuse = 0;
  int old_ngrp = -1;
  for (size_t c = 0; c < cands.size(); ++c) {
    Plan &p = cands[c].plan;
    const bool recount = (c == 0) || p.n_grp != old_ngrp;
    uint64_t mbytes = 0, mops = 0;
    if (recount) {
      old_ngrp = p.n_grp;
      cbytes = 0;
      cops = 0;
    }
    for (int g = 0; g < p.n_grp; ++g) {
      const Group &gp = p.grp[g];
      if (recount) last = counts_for(gp);
      if (gp.n_imten != 0)
        reuse = (g < p.n_grp - 1) ? p.grp[g + 1].memo_mode - gp.memo_mode - 1
                                  : (uint64_t)N - gp.memo_mode - 1;
      if (recount) {
        cbytes += csf_bytes(last);
        cops += csf_ops(last);
      }
      mbytes += memo_bytes(gp, last);
      mops += memo_ops(gp, reuse, last);
    }
    cands[c].pspace = cbytes + mbytes;
    cands[c].pops = cops + mops;
  }
}

void plan_features(const DevCoo &coo, uint64_t R, const std::vector<Candidate> &cands,
                   std::vector<float> &features, std::vector<double> &bytes, cudaStream_t s) {
  const int N = coo.nmodes;
  const double nnz = (double)std::max<uint64_t>(coo.nnz, 1);
  std::map<std::vector<uint64_t>, std::vector<uint64_t>> cache;
  auto counts_for = [&](const Group &g) {
    std::vector<uint64_t> key(g.o_opt, g.o_opt + N);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    std::vector<uint64_t> nf(N, 0);
    csf_count(coo, g.o_opt, nf.data(), s);
    nf[N - 1] = coo.nnz;
    cache[key] = nf;
    return nf;
  };
  double ldmean = 0, ldmax = -1e30, ldmin = 1e30;
  for (int m = 0; m < N; ++m) {
    const double ld = std::log10((double)std::max<uint64_t>(coo.dims[m], 1));
    ldmean += ld / N;
    ldmax = std::max(ldmax, ld);
    ldmin = std::min(ldmin, ld);
  }
  features.assign(cands.size() * kPlanFeatures, 0.f);
  bytes.assign(cands.size(), 0.0);
  for (size_t c = 0; c < cands.size(); ++c) {
    Plan p = cands[c].plan;
    decide_use_csfs(p);
    std::vector<std::vector<uint64_t>> nf(p.n_csf);
    double tree_nodes = 0, space = 0;
    for (int g = 0; g < p.n_csf; ++g) {
      nf[g] = counts_for(p.tree(g));
      for (int l = 0; l < N; ++l) tree_nodes += (double)nf[g][l];
      space += 9.0 * nnz;  // leaf ids, FP32 + FP64 values, close depths
      for (int l = 0; l < N - 1; ++l) space += 9.0 * (double)nf[g][l];
      for (uint64_t d = 0; d < p.tree(g).n_imten; ++d)
        space += 4.0 * (double)ldr_of((int)R) * (double)nf[g][p.tree(g).begin_imten - 1 - d];
    }
    // the walk of every mode, as the engine builds it: source level S,
    // output level d (the mode's depth), stored levels
    double cu = 0, su = 0, items = 0, stored = 0, fan = 0;
    int n_leaf = 0, n_rows = 0, n_scatter = 0;
    for (int m = 0; m < N; ++m) {
      const int g = (int)p.use_csfs[m];
      const Group &gp = p.tree(g);
      int d = 0;
      for (int l = 0; l < N; ++l)
        if ((int)gp.o_opt[l] == m) d = l;
      int S = N - 1;
      if (p.use_tags[m] == 0 && gp.n_imten > 0) {
        for (uint64_t deg = 0; deg < gp.n_imten; ++deg)
          stored += (double)nf[g][gp.begin_imten - 1 - deg];
      } else if (p.use_tags[m] == 1) {
        // mttkrp.c:1578-1588 with rcsf_reverse_mode_order (adatm_rcsf.c:313-326)
        const uint64_t b = gp.begin_imten;
        uint64_t rd[kMaxModes + 1] = {0};
        uint64_t j = 0;
        for (int64_t i = (int64_t)b; i >= 0; --i)
          if (i != d) rd[j++] = (uint64_t)i;
        uint64_t indeg = 0;
        for (uint64_t i = 0; i < gp.n_imten; ++i)
          if (b - i == rd[i]) ++indeg;
        if (indeg > 0) S = (int)(b - indeg);
      }
      const double units = (double)nf[g][S];
      if (S == N - 1) ++n_leaf;
      else ++n_rows;
      if (S > d) {
        cu += units;
        for (int l = d; l < S; ++l) items += (double)nf[g][l];
      } else {
        su += units;
        ++n_scatter;
        fan += std::log10(1.0 + units / (double)std::max<uint64_t>(coo.dims[m], 1));
      }
    }
    float *x = &features[c * kPlanFeatures];
    x[0] = (float)N;
    x[1] = (float)std::log10(nnz);
    x[2] = (float)std::log2((double)R);
    x[3] = (float)ldmean;
    x[4] = (float)ldmax;
    x[5] = (float)ldmin;
    x[6] = (float)p.n_grp;
    x[7] = (float)std::log10(1.0 + cu);
    x[8] = (float)std::log10(1.0 + su);
    x[9] = (float)(items / nnz);
    x[10] = (float)(stored / nnz);
    x[11] = (float)n_leaf / N;
    x[12] = (float)n_rows / N;
    x[13] = (float)n_scatter / N;
    x[14] = (float)(tree_nodes / nnz);
    x[15] = (float)(n_scatter ? fan / n_scatter : 0.0);
    bytes[c] = space;
  }
}

int choose_candidate(const std::vector<Candidate> &cands, int strategy, double slimit) {
  std::vector<int> fit;
  for (size_t c = 0; c < cands.size(); ++c)
    if ((double)cands[c].pspace < slimit) fit.push_back((int)c);
  if (fit.empty()) return -1;
  int best = 0;
  for (size_t c = 1; c < fit.size(); ++c) {
    const Candidate &x = cands[fit[c]], &b = cands[fit[best]];
    if (strategy == 2 ? x.pspace < b.pspace : x.pops < b.pops) best = (int)c;
  }
  // the reference hands back the position in the filtered list and indexes
  // the full list with it (adatm_bench.c:482-485)
  return best;
}

Plan plan_analytic(const DevCoo &coo, uint64_t R, int strategy, std::vector<Candidate> *all,
                   cudaStream_t s) {
  std::vector<Candidate> c = candidate_configs(coo.nmodes, coo.dims);
  predict_candidates(coo, R, c, s);
  const int pick = choose_candidate(c, strategy, 90e9);
  if (all) *all = c;
  if (pick < 0) throw NoMemory("no memoization plan fits the storage limit");
  Plan p = c[pick].plan;
  decide_use_csfs(p);
  return p;
}

namespace {
// locate_ind_special (adatm_utils.c:9-29): position of ele among the memo
// modes, x.5 between two of them, -1 if none. The reference's loop stops
// after its first pass (the `break` at :23), so only positions 0 and 1 and
// the tail are ever found; that behaviour is kept, it decides the plan.
double locate_ind_special(const uint64_t *array, uint64_t length, uint64_t ele, uint64_t nmodes) {
  double loc = -1;
  if (array[0] == ele) loc = 0;
  for (uint64_t i = 1; i < length; ++i) {
    if (array[i] == ele) loc = (double)i;
    else if (array[i - 1] < ele && ele < array[i]) loc = (double)i - 0.5;
    break;
  }
  if (array[length - 1] < ele && ele < nmodes) loc = (double)length - 0.5;
  return loc;
}
}  // namespace

void decide_use_csfs_space(Plan &p) {
  const int N = p.nmodes;
  int memo_groups[kMaxModes];
  uint64_t csf_modes[kMaxModes];
  int n = 0;
  for (int g = 0; g < p.n_grp; ++g)
    if (p.grp[g].n_imten > 0) {
      memo_groups[n] = g;
      csf_modes[n] = p.grp[g].memo_mode;
      ++n;
    }
  if (p.n_grp == 1 || n == 0 || n == p.n_grp) {
    decide_use_csfs(p);
    return;
  }
  p.space_efficient = true;
  p.n_csf = n;
  for (int t = 0; t < kMaxModes; ++t) p.tree_group[t] = t < n ? memo_groups[t] : 0;
  // mttkrp.c:1976-2029. Modes the reference leaves unassigned (its
  // locate_ind_special misses them) recompute on tree 0.
  bool set[kMaxModes] = {false};
  auto assign = [&](uint64_t first, uint64_t stop, double loc) {
    if (loc < 0) return;
    const uint64_t t = (uint64_t)loc;
    const bool exact = loc - (double)t == 0;
    p.use_csfs[first] = t;
    p.use_tags[first] = exact ? 0 : 2;
    set[first] = true;
    for (uint64_t rm = first + 1; rm < stop; ++rm) {
      p.use_csfs[rm] = t;
      p.use_tags[rm] = exact ? 1 : 2;
      set[rm] = true;
    }
  };
  for (int g = 0; g + 1 < p.n_grp; ++g) {
    const uint64_t mode = p.grp[g].memo_mode;
    assign(mode, p.grp[g + 1].memo_mode, locate_ind_special(csf_modes, n, mode, N));
    const uint64_t last = p.grp[p.n_grp - 1].memo_mode;
    assign(last, (uint64_t)N, locate_ind_special(csf_modes, n, last, N));
  }
  for (int m = 0; m < N; ++m)
    if (!set[m]) {
      p.use_csfs[m] = 0;
      p.use_tags[m] = 2;
    }
}

void decide_use_csfs(Plan &p) {
  // TIME_EFFICIENT: one tree per group (mttkrp.c:1956-1975)
  const int N = p.nmodes;
  p.n_csf = p.n_grp;
  p.space_efficient = false;
  for (int t = 0; t < kMaxModes; ++t) p.tree_group[t] = t;
  for (int g = 0; g < p.n_grp; ++g) {
    const uint64_t mode = p.grp[g].memo_mode;
    const uint64_t stop = (g + 1 < p.n_grp) ? p.grp[g + 1].memo_mode : (uint64_t)N;
    p.use_csfs[mode] = (uint64_t)g;
    p.use_tags[mode] = 0;
    for (uint64_t rm = mode + 1; rm < stop; ++rm) {
      p.use_csfs[rm] = (uint64_t)g;
      p.use_tags[rm] = 1;
    }
  }
}

void splatt_perm(int nmodes, const uint64_t *dims, bool root_first, uint64_t root, uint64_t *perm) {
  int k = 0;
  bool used[kMaxModes] = {false};
  if (root_first) {
    perm[k++] = root;
    used[root] = true;
  }
  while (k < nmodes) {
    int best = -1;
    for (int m = 0; m < nmodes; ++m)
      if (!used[m] && (best < 0 || dims[m] < dims[best])) best = m;
    used[best] = true;
    perm[k++] = (uint64_t)best;
  }
}

Plan plan_splatt(int nmodes, const uint64_t *dims, int csf_alloc) {
  Plan p;
  p.nmodes = nmodes;
  if (csf_alloc == 2) {  // ALLMODE
    p.n_grp = nmodes;
    p.n_csf = nmodes;
    for (int m = 0; m < nmodes; ++m) {
      p.grp[m].memo_mode = (uint64_t)m;
      p.grp[m].begin_imten = 1;
      p.grp[m].n_imten = 0;
      splatt_perm(nmodes, dims, true, (uint64_t)m, p.grp[m].o_opt);
      p.use_csfs[m] = (uint64_t)m;
      p.use_tags[m] = 0;
    }
    return p;
  }
  uint64_t order[kMaxModes];
  splatt_perm(nmodes, dims, false, 0, order);
  p.grp[0].memo_mode = order[0];
  p.grp[0].begin_imten = 1;
  p.grp[0].n_imten = 0;
  for (int l = 0; l < nmodes; ++l) p.grp[0].o_opt[l] = order[l];
  p.n_grp = 1;
  p.n_csf = 1;
  for (int m = 0; m < nmodes; ++m) {
    p.use_csfs[m] = 0;
    p.use_tags[m] = ((uint64_t)m == order[0]) ? 0 : 2;
  }
  if (csf_alloc == 1) {  // TWOMODE: the largest mode through its own tree
    const uint64_t big = order[nmodes - 1];
    p.n_grp = 2;
    p.n_csf = 2;
    p.grp[1].memo_mode = big;
    p.grp[1].begin_imten = 1;
    p.grp[1].n_imten = 0;
    splatt_perm(nmodes, dims, true, big, p.grp[1].o_opt);
    p.use_csfs[big] = 1;
    p.use_tags[big] = 0;
  }
  return p;
}

}  // namespace adatm
