// mttkrp.cuh -- the MTTKRP kernels on CSF trees and their launch plans.
//
// Every MTTKRP of the reference (plain root / internal / leaf, memo root,
// memo reuse; mttkrp.c:241-1682) is one of two tree walks over a source
// level S and an output level d of one CSF tree:
//
//  * contract (S > d): every unit of level S (a nonzero when S = N-1, else a
//    stored memo row T_S) is multiplied by its factor row and summed into its
//    level S-1 parent; a completed node of level l > d multiplies its sum by
//    its own factor row and adds it to its parent; a completed node of level
//    d is written to the output row fids[d][node], multiplied by the prefix
//    product P_{d-1} of the factor rows on its root path (d > 0). Completed
//    nodes of the levels listed in `store` are also written to memo rows.
//  * scatter (S == d): every unit u adds src(u) * P_{d-1} to output row
//    fids[d][u] (leaf MTTKRP when d = N-1, memo reuse at its stored level).
//
// Work is split into chunks of `chunk` consecutive source units, one chunk
// per row group of LANES lanes (each lane holds 4 of the R columns), so the
// split follows nonzeros, not root slices (the reference's omp
// schedule(dynamic,16) over slices, mttkrp.c:392, cannot balance a slice
// holding 16% of the nonzeros). Nodes cut by a chunk boundary are combined
// with vector atomics; for memo rows those nodes are zeroed first by a
// separate launch, all other memo rows are written exactly once.
#pragma once

#include "csf_build.cuh"

namespace adatm {

enum class FactorType : int { F32 = 0, BF16 = 1 };

// Factor row matrices of one tree, in level order (U[l] belongs to mode
// dim_perm[l]); fp32 or bf16 with leading dimension ldr.
struct LevelFactors {
  const void *U[kMaxModes] = {nullptr};
};

struct TreeWalk {
  int nmodes = 0;
  int src = 0;                 // source level S
  int out = 0;                 // output level d
  int R = 0, ldr = 0;
  uint32_t chunk = 32;
  uint32_t nchunks = 0;
  uint64_t nunits = 0;         // nodes of level S
  const DevCsf *csf = nullptr;
  const float *src_rows = nullptr;           // memo rows of level S (S < N-1)
  float *store[kMaxModes] = {nullptr};       // memo rows written, per level
  DevBuf<uint32_t> sched;                    // nchunks x (S + 1), then the chunk counter
  bool resident = true;                      // contraction grid: resident blocks that claim
                                             // chunks (else one chunk per warp)
  int walkers = 0;                           // contraction source loop: walkers per warp
                                             // (1, 2 or 4; 0 = default_walkers(R))
  int fold = -1;                             // contraction: unstored levels below the
                                             // source folded into its loop (0..2; -1 =
                                             // chosen from the tree's fan-out)
  // Scatter walks: the output rows that the most units hit (at most
  // kHotRows, each hit by at least kHotMin units) are summed per block in
  // shared memory; hot_slot maps an output row to its slot (0xFF = none).
  int nhot = 0;
  DevBuf<uint8_t> hot_slot;
  DevBuf<uint32_t> hot_rows;
  // Nodes that chunk boundaries cut (contractions, every mode): their
  // partial sums go to per-chunk rows (span) and are summed per node in
  // chunk order and in FP64 (chains, in groups of kChainGroup partials), so
  // a node spanning thousands of chunks (a skewed root slice) takes no long
  // chain of FP32 atomics. Deterministic accumulation additionally pulls
  // scatters, and the output of contractions below the root, per output row
  // in the order of a stable sort by output row (segments of whole rows, long
  // rows split into pieces summed in order): no float atomics anywhere, so
  // repeated runs agree bit for bit.
  bool deterministic = false;
  int span_nlev = 0;
  int span_lev[kMaxModes] = {-1, -1, -1, -1, -1, -1, -1, -1};
  DevBuf<float> span;                // nchunks x span_nlev x 2 x ldr
  DevBuf<uint32_t> chains;           // per chain: level, node, first boundary chunk, last chunk,
                                     // first group, groups
  DevBuf<uint32_t> groups;           // per group: chain, first partial, partials
  DevBuf<double> gsum;               // per group: its sum (ldr)
  uint32_t nchains = 0, ngroups = 0;
  DevBuf<uint32_t> chain_ids;        // chains of few groups first (nshort), then long ones
  uint32_t nshort = 0;
  DevBuf<float> level_rows;          // contraction below the root: level-d node sums
  // pull scatter of level `out` (deterministic scatters and contractions below the root)
  bool pull = false;
  DevBuf<uint32_t> parent[kMaxModes];  // parent node of every node of levels 1..out
  DevBuf<uint32_t> perm, prow, pparent;  // units sorted by output row (stable), their rows, parents
  DevBuf<uint32_t> segs;             // per segment: first, end, piece slot (~0u: whole rows)
  DevBuf<uint32_t> pieces;           // per long row: row, first piece slot, pieces
  DevBuf<double> piece_sum;          // per piece: its sum (ldr)
  uint32_t nsegs = 0, nlong = 0, npieces = 0;
  DevBuf<float> prefix[2];           // prefix rows of levels 0..out-1 (ping-pong)
  bool has_store() const {
    for (int l = 0; l < kMaxModes; ++l)
      if (store[l]) return true;
    return false;
  }
};

// Kernel launches of one walk (for launch counts).
int walk_kernels(const TreeWalk &w);

// Walkers per warp of the contraction's source loop by default at rank R,
// and whether W walkers are built for rank R.
int default_walkers(int R);
bool walkers_supported(int R, int W);

// Fill the chunk schedule: node ids at levels 0..S-1 of every chunk's first
// unit, plus a bit mask of the levels whose node began before the chunk.
void walk_prepare(TreeWalk &w, cudaStream_t s);

// Launch the walk: output rows (FP64, dims x ldr) must be zero beforehand
// (the caller clears them).
void walk_launch(const TreeWalk &w, const LevelFactors &f, FactorType ft, double *out,
                 cudaStream_t s);

// Bytes the walk must move through HBM (structure read once, memo rows read
// or written once, factors read once, output written once): the compulsory
// traffic used for the roofline figure.
double walk_compulsory_bytes(const TreeWalk &w, FactorType ft, const uint64_t *dims_of_level,
                             uint64_t out_rows);

}  // namespace adatm
