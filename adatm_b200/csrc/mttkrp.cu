// mttkrp.cu -- tree-walk MTTKRP kernels (see mttkrp.cuh for the scheme).
#include <algorithm>
#include <type_traits>
#include <vector>

#include "mttkrp.cuh"

namespace adatm {

namespace {

struct WalkArgs {
  int N, S, d, R, ldr;
  uint32_t chunk, nchunks;
  uint64_t nunits;
  uint64_t nfibs[kMaxModes];
  const uint32_t *fptr[kMaxModes];
  const uint32_t *fids[kMaxModes];
  const float *vals;
  const float *src_rows;       // memo rows of the source level (S < N-1)
  const uint32_t *src_ids;     // fids of the source level
  const uint8_t *src_cd;       // close depths of the source level (S >= 1)
  const void *U_src;           // factor rows of the source level
  const void *U[kMaxModes];
  float *store[kMaxModes];
  double *out;                 // MTTKRP output rows (FP64 sums)
  const uint32_t *sched;
  uint32_t *counter;           // chunks claimed so far (zeroed before each launch)
  const uint8_t *hot_slot;     // scatter: slot of an output row summed per block, 0xFF = none
  const uint32_t *hot_rows;    // scatter: output row of each slot
  int nhot;
  // deterministic contraction: instead of atomics, the partial sums of the
  // nodes a chunk boundary cuts go to per-chunk rows (head: the node that
  // began before the chunk and closes in it; tail: the node open at its
  // end), summed later in chunk order; span_lev[l] is level l's slot
  // (-1 = none)
  float *span;
  int span_nlev;
  int span_lev[kMaxModes];
};

// Row of chunk c's head (which = 0) or tail (which = 1) partial at level l.
__device__ __forceinline__ float *span_row(const WalkArgs &a, uint32_t c, int l, int which) {
  return a.span + (((size_t)c * a.span_nlev + a.span_lev[l]) * 2 + which) * a.ldr;
}

constexpr int kHotRows = 32;     // output rows summed per block, at most
constexpr uint32_t kHotMin = 32768;  // units that must hit a row to make it one
constexpr uint64_t kHotScanRows = 1ull << 24;  // output rows the hot-row search examines, at most

// ---------------------------------------------------------------------------
// Warp-uniform tree walk.
//
// One warp walks one chunk of consecutive source units; its 32 lanes split
// the R columns (V = 1, 2 or 4 columns per lane), so every lane follows the
// same control flow and each factor-row gather is one coalesced access. Units
// go in batches of 32 (one per lane for the index loads): the batch's factor
// rows are gathered with many loads in flight, then summed in order into the
// open node of level S-1. Where a node closes is read from the tree's close
// depths (no fptr traffic): a unit with close depth c closes its ancestors at
// levels S-1 .. S-c. The nodes of level S-1 that close in the batch become
// the items of the next level up -- their sums sit in shared memory, are
// multiplied by their own factor rows and summed into level S-2 nodes in the
// same way -- until level d, where completed nodes go to the output.
// ---------------------------------------------------------------------------
constexpr int kWarps = 8;   // warps (chunks) per block
constexpr int kBatch = 32;  // source units per batch

template <int V>
struct alignas(sizeof(float) * V) fv {
  float x[V];
};

template <int V>
__device__ __forceinline__ fv<V> fv_fill(float s) {
  fv<V> r;
#pragma unroll
  for (int i = 0; i < V; ++i) r.x[i] = s;
  return r;
}
template <int V>
__device__ __forceinline__ void fv_axpy(fv<V> &acc, float s, const fv<V> &b) {
#pragma unroll
  for (int i = 0; i < V; ++i) acc.x[i] = fmaf(s, b.x[i], acc.x[i]);
}
template <int V>
__device__ __forceinline__ void fv_fma(fv<V> &acc, const fv<V> &a, const fv<V> &b) {
#pragma unroll
  for (int i = 0; i < V; ++i) acc.x[i] = fmaf(a.x[i], b.x[i], acc.x[i]);
}
template <int V>
__device__ __forceinline__ fv<V> fv_mul(const fv<V> &a, const fv<V> &b) {
  fv<V> r;
#pragma unroll
  for (int i = 0; i < V; ++i) r.x[i] = a.x[i] * b.x[i];
  return r;
}
template <int V>
__device__ __forceinline__ fv<V> fv_scale(float s, const fv<V> &a) {
  fv<V> r;
#pragma unroll
  for (int i = 0; i < V; ++i) r.x[i] = s * a.x[i];
  return r;
}

// Columns col..col+V-1 of factor row `row` (FP32 or BF16 storage).
template <int V, FactorType FT>
__device__ __forceinline__ fv<V> ld_factor(const void *U, uint32_t row, int ldr, int col, bool act) {
  fv<V> r = fv_fill<V>(0.f);
  if (!act) return r;
  if constexpr (FT == FactorType::F32) {
    const float *p = static_cast<const float *>(U) + (size_t)row * ldr + col;
    if constexpr (V == 1) {
      r.x[0] = __ldg(p);
    } else if constexpr (V == 2) {
      const float2 t = __ldg(reinterpret_cast<const float2 *>(p));
      r.x[0] = t.x;
      r.x[1] = t.y;
    } else {
      const float4 t = __ldg(reinterpret_cast<const float4 *>(p));
      r.x[0] = t.x;
      r.x[1] = t.y;
      r.x[2] = t.z;
      r.x[3] = t.w;
    }
  } else {
    const __nv_bfloat16 *p = static_cast<const __nv_bfloat16 *>(U) + (size_t)row * ldr + col;
    if constexpr (V == 1) {
      r.x[0] = __bfloat162float(__ldg(p));
    } else if constexpr (V == 2) {
      const float2 t = __bfloat1622float2(__ldg(reinterpret_cast<const __nv_bfloat162 *>(p)));
      r.x[0] = t.x;
      r.x[1] = t.y;
    } else {
      const uint2 raw = __ldg(reinterpret_cast<const uint2 *>(p));
      const float2 lo = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&raw.x));
      const float2 hi = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&raw.y));
      r.x[0] = lo.x;
      r.x[1] = lo.y;
      r.x[2] = hi.x;
      r.x[3] = hi.y;
    }
  }
  return r;
}

// FP32 row matrices (memo rows, outputs).
template <int V>
__device__ __forceinline__ fv<V> ld_rows(const float *base, uint64_t row, int ldr, int col, bool act) {
  fv<V> r = fv_fill<V>(0.f);
  if (!act) return r;
  const float *p = base + row * (uint64_t)ldr + col;
  if constexpr (V == 1) {
    r.x[0] = __ldg(p);
  } else if constexpr (V == 2) {
    const float2 t = __ldg(reinterpret_cast<const float2 *>(p));
    r.x[0] = t.x;
    r.x[1] = t.y;
  } else {
    const float4 t = __ldg(reinterpret_cast<const float4 *>(p));
    r.x[0] = t.x;
    r.x[1] = t.y;
    r.x[2] = t.z;
    r.x[3] = t.w;
  }
  return r;
}

template <int V>
__device__ __forceinline__ void st_rows(float *base, uint64_t row, int ldr, int col, const fv<V> &v,
                                        bool act) {
  if (!act) return;
  float *p = base + row * (uint64_t)ldr + col;
  if constexpr (V == 1) {
    *p = v.x[0];
  } else if constexpr (V == 2) {
    *reinterpret_cast<float2 *>(p) = make_float2(v.x[0], v.x[1]);
  } else {
    *reinterpret_cast<float4 *>(p) = make_float4(v.x[0], v.x[1], v.x[2], v.x[3]);
  }
}

template <int V>
__device__ __forceinline__ void red_rows(float *base, uint64_t row, int ldr, int col, const fv<V> &v,
                                         bool act) {
  if (!act) return;
  float *p = base + row * (uint64_t)ldr + col;
  if constexpr (V == 1) {
    atomicAdd(p, v.x[0]);
  } else if constexpr (V == 2) {
    atomicAdd(reinterpret_cast<float2 *>(p), make_float2(v.x[0], v.x[1]));
  } else {
    atomicAdd(reinterpret_cast<float4 *>(p), make_float4(v.x[0], v.x[1], v.x[2], v.x[3]));
  }
}

// FP64 output rows: the MTTKRP sums of a row can come from millions of
// units (a skewed slice), and FP32 sums of that many partials lose several
// digits; outputs are stored and added in FP64.
template <int V>
__device__ __forceinline__ void st_out(double *base, uint64_t row, int ldr, int col, const fv<V> &v,
                                       bool act) {
  if (!act) return;
  double *p = base + row * (uint64_t)ldr + col;
  if constexpr (V == 1) {
    *p = v.x[0];
  } else if constexpr (V == 2) {
    *reinterpret_cast<double2 *>(p) = make_double2(v.x[0], v.x[1]);
  } else {
    *reinterpret_cast<double2 *>(p) = make_double2(v.x[0], v.x[1]);
    *reinterpret_cast<double2 *>(p + 2) = make_double2(v.x[2], v.x[3]);
  }
}

template <int V>
__device__ __forceinline__ void red_out(double *base, uint64_t row, int ldr, int col, const fv<V> &v,
                                        bool act) {
  if (!act) return;
  double *p = base + row * (uint64_t)ldr + col;
#pragma unroll
  for (int i = 0; i < V; ++i) atomicAdd(p + i, (double)v.x[i]);
}

// Factor-row gathers through a per-lane base pointer (the lane's first
// column) and a byte stride, so an address is one wide multiply-add.
template <int V, FactorType FT>
struct RowSrc {
  const char *base = nullptr;
  uint32_t stride = 0;
  // Lanes past the rank read column 0 (their results are never stored).
  __device__ __forceinline__ RowSrc(const void *U, int ldr, int col, bool act) {
    constexpr int esz = FT == FactorType::F32 ? 4 : 2;
    base = static_cast<const char *>(U) + (size_t)(act ? col : 0) * esz;
    stride = (uint32_t)ldr * esz;
  }
  // Row `row`, or row 0 when !on: the load is always issued at a valid
  // address, so no branch splits a batch of loads.
  __device__ __forceinline__ fv<V> load(uint32_t row, bool on) const {
    fv<V> r;
    const char *p = base + (size_t)(on ? row : 0u) * stride;
    if constexpr (FT == FactorType::F32) {
      if constexpr (V == 1) {
        r.x[0] = __ldg(reinterpret_cast<const float *>(p));
      } else if constexpr (V == 2) {
        const float2 t = __ldg(reinterpret_cast<const float2 *>(p));
        r.x[0] = t.x;
        r.x[1] = t.y;
      } else {
        const float4 t = __ldg(reinterpret_cast<const float4 *>(p));
        r.x[0] = t.x;
        r.x[1] = t.y;
        r.x[2] = t.z;
        r.x[3] = t.w;
      }
    } else {
      if constexpr (V == 1) {
        r.x[0] = __bfloat162float(__ldg(reinterpret_cast<const __nv_bfloat16 *>(p)));
      } else if constexpr (V == 2) {
        const float2 t = __bfloat1622float2(__ldg(reinterpret_cast<const __nv_bfloat162 *>(p)));
        r.x[0] = t.x;
        r.x[1] = t.y;
      } else {
        const uint2 raw = __ldg(reinterpret_cast<const uint2 *>(p));
        const float2 lo = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&raw.x));
        const float2 hi = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&raw.y));
        r.x[0] = lo.x;
        r.x[1] = lo.y;
        r.x[2] = hi.x;
        r.x[3] = hi.y;
      }
    }
    return r;
  }
};

// Shared memory of one contraction warp: kBatch item rows and one row per
// level 0..N-2 -- the prefix P_l = U_0[node_0] * ... * U_l[node_l] for l < d,
// the open node's partial sum (carry) for d <= l < S; the two ranges never
// overlap -- all in fv<V> slots of 32 lanes; then the batch's (id, value)
// (and parent) words and a 32-word exchange buffer.
template <int V>
__host__ __device__ constexpr size_t contract_warp_smem(int N) {
  return (size_t)(kBatch + N - 1) * 32 * sizeof(fv<V>) +
         (kBatch + kBatch / 16) * sizeof(uint4) + kBatch * sizeof(uint32_t);
}
// Staging slot of batch unit k: one spare uint4 every 16 units, so the two
// or four walkers of a warp reading units 16 apart hit different banks.
__device__ __forceinline__ int ustage_slot(int k) { return k + (k >> 4); }
template <int V>
constexpr size_t contract_smem(int N) {
  return (size_t)kWarps * contract_warp_smem<V>(N);
}

// Recompute the prefix rows of levels lo..hi-1 from the node indices (lane l
// of nodeL holds the node of level l).
template <int V, FactorType FT>
__device__ __noinline__ void refresh_prefix(const WalkArgs &a, fv<V> *pre, uint32_t nodeL, int lo,
                                            int hi, int col, bool act, int lane) {
  for (int l = lo; l < hi; ++l) {
    const uint32_t n = __shfl_sync(~0u, nodeL, l);
    const bool valid = (uint64_t)n < a.nfibs[l];
    const uint32_t f = valid ? __ldg(a.fids[l] + n) : 0u;
    const fv<V> row = ld_factor<V, FT>(a.U[l], f, a.ldr, col, act && valid);
    pre[l * 32 + lane] = l == 0 ? row : fv_mul(pre[(l - 1) * 32 + lane], row);
  }
}

// Levels lo..hi-1 move on to their next node (their nodes closed); their
// prefix rows are recomputed. Returns the updated per-lane node register.
template <int V, FactorType FT>
__device__ __noinline__ uint32_t advance_prefix(const WalkArgs &a, fv<V> *pre, uint32_t nodeL,
                                                int lo, int hi, int col, bool act, int lane) {
  if (lane >= lo && lane < hi) nodeL += 1;
  if (lo < hi && (uint64_t)__shfl_sync(~0u, nodeL, lo) < a.nfibs[lo])
    refresh_prefix<V, FT>(a, pre, nodeL, lo, hi, col, act, lane);
  return nodeL;
}

// Compaction of per-lane values onto the set bits of m: lane i gets the
// value of the lane holding the i-th set bit (i < popc(m)), else 0.
__device__ __forceinline__ uint32_t compact_bits(uint32_t m, uint32_t value, uint32_t *xbuf, int lane) {
  if ((m >> lane) & 1u) xbuf[__popc(m & lanemask_lt())] = value;
  __syncwarp();
  const uint32_t r = lane < __popc(m) ? xbuf[lane] : 0u;
  __syncwarp();
  return r;
}

// Contraction (S > d).
//
// The source units of a batch are summed into the open node of level S-1
// (carry `acc`, in registers); the level-(S-1) nodes that close become the
// batch's items. The level loop then takes the items up one level at a time
// -- memo stores, the items' own factor rows, carries of the levels above in
// shared memory -- until level d. Resident blocks per SM follow the shared
// memory a block takes (4 at V = 1, so at most 64 registers per thread).
template <int V>
constexpr int contract_min_blocks() {
  return V == 1 ? 4 : (V == 2 ? 2 : 1);
}

//
// FOLD F (levels S-1 .. S-F are not stored and lie below d): the nodes of
// those levels are not formed. Each unit's product is multiplied by the
// factor rows of its ancestors at levels S-1 .. S-F (U_{S-1} of the
// level-(S-1) node holding it, and at F = 2 U_{S-2} of the level-(S-2) node
// holding that) and summed straight into the open node of level S-1-F, so
// the batch's items are level-(S-1-F) nodes. The ancestors of a batch's
// units are consecutive nodes from each level's open node on (a unit's is
// the open node plus the closes of that level before it), so their ids come
// with one coalesced load per level. Folding trades one item of level l for
// one extra gather per unit below it: it pays where levels are hypersparse
// (few units per node). The sums equal the unfolded ones up to FP32
// rounding order.
// WALKERS: the source loop of a batch runs as W walkers of 32/W lanes, each
// over its own contiguous segment of 32/W units with VW columns per lane, so
// one warp instruction advances W units. Each walker sums its segment into
// its own open node; the nodes that close in a walker's segment become items
// as before, and the segments are joined once per batch: the sum a walker
// carries past its segment flows into the next walker's first closed node
// (or on through, when that walker closes none), W - 1 shuffle rounds. The
// level loop keeps the warp-wide layout (V columns per lane); items and
// carry rows are plain column-ordered rows in shared memory, so both
// layouts read them.
template <int V, int W, int VW, FactorType FT, bool LEAF, int F>
__global__ void __launch_bounds__(256, contract_min_blocks<V>())
    k_contract(const __grid_constant__ WalkArgs a) {
  static_assert(F >= 0 && F <= 2, "folded levels");
  static_assert(W == 1 || W == 2 || W == 4, "walkers per warp");
  static_assert((32 / W) * VW <= 32 * V, "a walker's columns must fit the item rows");
  constexpr int L = 32 / W;        // lanes per walker
  constexpr int SEG = kBatch / W;  // units per walker per batch
  extern __shared__ __align__(16) unsigned char walk_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char *wbase = walk_raw + (size_t)warp * contract_warp_smem<V>(a.N);
  fv<V> *items = reinterpret_cast<fv<V> *>(wbase);
  float *items_f = reinterpret_cast<float *>(wbase);  // row j: 32 * V floats
  fv<V> *carry = items + kBatch * 32;  // rows d..S-1
  fv<V> *pre = carry;                  // rows 0..d-1
  uint4 *ustage = reinterpret_cast<uint4 *>(carry + (a.N - 1) * 32);
  uint32_t *xbuf = reinterpret_cast<uint32_t *>(ustage + kBatch + kBatch / 16);
  const int col = lane * V;
  const bool act = col < a.R;
  const int wk = lane / L;           // this lane's walker
  const int wcol = (lane % L) * VW;  // its first column in the walker layout
  const bool wact = wcol < a.R;
  const int S = a.S, d = a.d;
  // a resident grid: each warp claims chunks from a counter, the next one
  // while it walks the current one; without a counter, one chunk per warp
  const bool claims = a.counter != nullptr;
  uint32_t claim = claims && lane == 0 ? atomicAdd(a.counter, 1u) : 0u;
  uint32_t chunk_id = claims ? __shfl_sync(~0u, claim, 0) : blockIdx.x * kWarps + warp;
  while (chunk_id < a.nchunks) {
    if (claims && lane == 0) claim = atomicAdd(a.counter, 1u);
    const uint32_t *sc = a.sched + (size_t)chunk_id * (S + 1);
    uint32_t nodeL = lane < S ? sc[lane] : 0u;
    uint32_t part = sc[S];
    uint32_t touched = 0;
    for (int l = d; l < S - 1; ++l) carry[l * 32 + lane] = fv_fill<V>(0.f);
    if (d > 0) refresh_prefix<V, FT>(a, pre, nodeL, 0, d, col, act, lane);
    const RowSrc<VW, FT> Us(a.U_src, a.ldr, wcol, wact);
    const RowSrc<VW, FT> Up(F >= 1 ? a.U[S - 1] : a.U_src, a.ldr, wcol, wact);
    const RowSrc<VW, FT> Uq(F >= 2 ? a.U[S - 2] : a.U_src, a.ldr, wcol, wact);
    const int top = S - 1 - F;  // level whose open node the units feed
    // open node of level `top` carried in from earlier batches (every walker
    // holds the same copy)
    fv<VW> acc = fv_fill<VW>(0.f);
    // unit rows in flight per lane, never more than the walker's segment:
    // fewer as each unit gathers more rows (the 64 registers a thread has at
    // four blocks per SM are the limit; spilling costs more than the extra
    // load latency exposed)
    constexpr int SB0 = (F == 2 ? 4 : (F == 1 ? 8 : 16)) / VW;
    constexpr int SB = SB0 < SEG ? SB0 : SEG;
    static_assert(SEG % SB == 0, "a walker's segment is a whole number of load groups");
    const uint64_t u0 = (uint64_t)chunk_id * a.chunk;
    const uint64_t u1 = min(u0 + a.chunk, a.nunits);
    for (uint64_t base = u0; base < u1; base += kBatch) {
      const int cnt = (int)min((uint64_t)kBatch, u1 - base);
      const bool in = lane < cnt;
      const uint32_t id = in ? __ldg(a.src_ids + base + lane) : 0u;
      float v = 0.f;
      if constexpr (LEAF) v = in ? __ldg(a.vals + base + lane) : 0.f;
      const uint32_t cd = in ? (uint32_t)__ldg(a.src_cd + base + lane) : 0u;
      const uint32_t M = __ballot_sync(~0u, cd >= 1u);
      uint32_t pfid = 0u, qfid = 0u, M2 = 0u;
      if constexpr (F >= 1) {
        // unit lane sits in level-(S-1) node first + (closes before it)
        const uint64_t pn = (uint64_t)__shfl_sync(~0u, nodeL, S - 1) + __popc(M & lanemask_lt());
        if (in && pn < a.nfibs[S - 1]) pfid = __ldg(a.fids[S - 1] + pn);
      }
      if constexpr (F >= 2) {
        // and in level-(S-2) node first + (level-(S-2) closes before it)
        M2 = __ballot_sync(~0u, cd >= 2u);
        const uint64_t qn = (uint64_t)__shfl_sync(~0u, nodeL, S - 2) + __popc(M2 & lanemask_lt());
        if (in && qn < a.nfibs[S - 2]) qfid = __ldg(a.fids[S - 2] + qn);
      }
      // closes of level `top`
      const uint32_t Mc = F == 0 ? M : (F == 1 ? __ballot_sync(~0u, cd >= 2u) : __ballot_sync(~0u, cd >= 3u));
      ustage[ustage_slot(lane)] = make_uint4(id, __float_as_uint(v), pfid, qfid);
      __syncwarp();
      // this walker's units are k_lo .. k_lo + SEG - 1: its closes, and the
      // item index of its first close
      const int k_lo = wk * SEG;
      const uint32_t below = k_lo == 0 ? 0u : (0xFFFFFFFFu >> (32 - k_lo));
      const uint32_t Mw = Mc & ((0xFFFFFFFFu >> (32 - SEG)) << k_lo);
      const int j0 = __popc(Mc & below);
      int j = j0;
      fv<VW> wacc = W == 1 ? acc : fv_fill<VW>(0.f);
      auto emit = [&](const fv<VW> &x) {
        *reinterpret_cast<fv<VW> *>(items_f + (size_t)j * 32 * V + wcol) = x;
        ++j;
      };
      auto run = [&](auto full) {
        constexpr bool FULL = decltype(full)::value;
#pragma unroll
        for (int q0 = 0; q0 < SEG; q0 += SB) {
          if (!FULL && k_lo + q0 >= cnt) break;
          fv<VW> g[SB];
          fv<VW> h[F >= 1 ? SB : 1];
          fv<VW> h2[F >= 2 ? SB : 1];
          fv<VW> m[LEAF ? 1 : SB];
          float vv[LEAF ? SB : 1];
#pragma unroll
          for (int q = 0; q < SB; ++q) {
            const int k = k_lo + q0 + q;
            // lanes past the rank read column 0 through Us's base, so only
            // the units past the batch need the row-0 substitute
            const bool ok = FULL || k < cnt;
            const uint4 e = ustage[ustage_slot(k)];
            g[q] = Us.load(e.x, ok);
            if constexpr (F >= 1) h[q] = Up.load(e.z, ok);
            if constexpr (F >= 2) h2[q] = Uq.load(e.w, ok);
            if constexpr (LEAF) vv[q] = __uint_as_float(e.y);
            if constexpr (!LEAF) m[q] = ld_rows<VW>(a.src_rows, base + k, a.ldr, wcol, ok && wact);
          }
#pragma unroll
          for (int q = 0; q < SB; ++q) {
            const int k = k_lo + q0 + q;
            if (FULL || k < cnt) {
              if constexpr (F >= 1) {
                fv<VW> x = LEAF ? fv_scale(vv[LEAF ? q : 0], g[q]) : fv_mul(m[LEAF ? 0 : q], g[q]);
                if constexpr (F >= 2) {
                  x = fv_mul(x, h[q]);
                  fv_fma(wacc, x, h2[F >= 2 ? q : 0]);
                } else {
                  fv_fma(wacc, x, h[F >= 1 ? q : 0]);
                }
              } else if constexpr (LEAF) {
                fv_axpy(wacc, vv[LEAF ? q : 0], g[q]);
              } else {
                fv_fma(wacc, m[LEAF ? 0 : q], g[q]);
              }
              if ((Mw >> k) & 1u) {
                emit(wacc);
                wacc = fv_fill<VW>(0.f);
              }
            }
          }
        }
      };
      if (cnt == kBatch) run(std::true_type{});
      else run(std::false_type{});
      if constexpr (W == 1) {
        acc = wacc;
      } else {
        // join the segments: the inflow of walker w is what walker w-1
        // carries past its segment (the carry-in for walker 0)
        const bool hc = Mw != 0u;
        fv<VW> inflow = acc, out;
#pragma unroll
        for (int i = 0; i < VW; ++i) out.x[i] = hc ? wacc.x[i] : inflow.x[i] + wacc.x[i];
#pragma unroll
        for (int r = 0; r + 1 < W; ++r) {
#pragma unroll
          for (int i = 0; i < VW; ++i) {
            const float up = __shfl_up_sync(~0u, out.x[i], L);
            if (wk == r + 1) {
              inflow.x[i] = up;
              out.x[i] = hc ? wacc.x[i] : up + wacc.x[i];
            }
          }
        }
        if (hc) {
          fv<VW> *first = reinterpret_cast<fv<VW> *>(items_f + (size_t)j0 * 32 * V + wcol);
          fv<VW> t = *first;
#pragma unroll
          for (int i = 0; i < VW; ++i) t.x[i] += inflow.x[i];
          *first = t;
        }
#pragma unroll
        for (int i = 0; i < VW; ++i) acc.x[i] = __shfl_sync(~0u, out.x[i], (W - 1) * L + lane % L);
      }
      __syncwarp();
      if ((Mc >> (cnt - 1)) & 1u) touched &= ~(1u << top);
      else touched |= 1u << top;
      if (F >= 1 && M != 0u) {
        if (lane == S - 1) nodeL += (uint32_t)__popc(M);
        part &= ~(1u << (S - 1));
      }
      if (F >= 2 && M2 != 0u) {
        if (lane == S - 2) nodeL += (uint32_t)__popc(M2);
        part &= ~(1u << (S - 2));
      }
      int n = __popc(Mc);
      uint32_t icd = compact_bits(Mc, cd - (uint32_t)(F + 1), xbuf, lane);
      // the level loop: items of level l (node sums that closed in this batch)
      for (int l = top; l >= d && n > 0; --l) {
        const uint32_t first = __shfl_sync(~0u, nodeL, l);
        const bool pfirst = (part >> l) & 1u;
        const uint32_t fid =
            (lane < n && (uint64_t)first + lane < a.nfibs[l]) ? __ldg(a.fids[l] + first + lane) : 0u;
        float *store = a.store[l];
        if (store != nullptr && (uint64_t)first + n <= a.nfibs[l]) {
          float *sp = store + (size_t)first * a.ldr + col;
          if (!pfirst) st_rows<V>(sp, 0, 0, 0, items[lane], act);
          else if (a.span) st_rows<V>(span_row(a, chunk_id, l, 0), 0, 0, col, items[lane], act);
          else red_rows<V>(sp, 0, 0, 0, items[lane], act);
          for (int i = 1; i < n; ++i) {
            sp += a.ldr;
            st_rows<V>(sp, 0, 0, 0, items[i * 32 + lane], act);
          }
        }
        if (l > d) {
          const uint32_t Mp = __ballot_sync(~0u, lane < n && icd >= 1u);
          const RowSrc<V, FT> Ul(a.U[l], a.ldr, col, act);
          fv<V> cl = carry[(l - 1) * 32 + lane];
          int jj = 0;
  #pragma unroll 8
          for (int i = 0; i < n; ++i) {
            const fv<V> row = Ul.load(__shfl_sync(~0u, fid, i), true);
            fv_fma(cl, items[i * 32 + lane], row);
            if ((Mp >> i) & 1u) {
              items[jj * 32 + lane] = cl;
              cl = fv_fill<V>(0.f);
              ++jj;
            }
          }
          carry[(l - 1) * 32 + lane] = cl;
          if ((Mp >> (n - 1)) & 1u) touched &= ~(1u << (l - 1));
          else touched |= 1u << (l - 1);
          if (lane == l) nodeL += (uint32_t)n;
          part &= ~(1u << l);
          icd = compact_bits(Mp, icd - 1u, xbuf, lane);
          n = __popc(Mp);
        } else {
          for (int i = 0; i < n; ++i) {
            const fv<V> val = items[i * 32 + lane];
            const uint32_t orow = __shfl_sync(~0u, fid, i);
            if (a.out == nullptr) {
              // deterministic d > 0: the level-d sums went to a store row
            } else if (d == 0) {
              if (!(i == 0 && pfirst)) st_out<V>(a.out, orow, a.ldr, col, val, act);
              else if (a.span) st_rows<V>(span_row(a, chunk_id, 0, 0), 0, 0, col, val, act);
              else red_out<V>(a.out, orow, a.ldr, col, val, act);
            } else {
              red_out<V>(a.out, orow, a.ldr, col, fv_mul(val, pre[(d - 1) * 32 + lane]), act);
              const uint32_t ci = __shfl_sync(~0u, icd, i);
              if (ci >= 1u) nodeL = advance_prefix<V, FT>(a, pre, nodeL, d - (int)ci, d, col, act, lane);
            }
          }
          if (lane == l) nodeL += (uint32_t)n;
          part &= ~(1u << l);
          n = 0;
        }
      }
    }
    // chunk end: the open nodes of levels top .. d add their partial sums
    // (the carried row, in the walker layout, is written by walker 0)
    if (wk == 0)
      *reinterpret_cast<fv<VW> *>(reinterpret_cast<float *>(carry) + (size_t)top * 32 * V + wcol) = acc;
    __syncwarp();
    for (int l = top; l >= d; --l) {
      if (!((touched >> l) & 1u)) continue;
      const uint32_t node = __shfl_sync(~0u, nodeL, l);
      if ((uint64_t)node >= a.nfibs[l]) continue;
      const fv<V> val = carry[l * 32 + lane];
      if (a.store[l] != nullptr) {
        if (a.span) st_rows<V>(span_row(a, chunk_id, l, 1), 0, 0, col, val, act);
        else red_rows<V>(a.store[l], node, a.ldr, col, val, act);
      }
      if (l > d) {
        const fv<V> r = ld_factor<V, FT>(a.U[l], __ldg(a.fids[l] + node), a.ldr, col, act);
        fv<V> c2 = carry[(l - 1) * 32 + lane];
        fv_fma(c2, val, r);
        carry[(l - 1) * 32 + lane] = c2;
        touched |= 1u << (l - 1);
      } else if (a.out != nullptr) {
        if (a.span && d == 0) {
          st_rows<V>(span_row(a, chunk_id, 0, 1), 0, 0, col, val, act);
        } else {
          const uint32_t orow = __ldg(a.fids[d] + node);
          red_out<V>(a.out, orow, a.ldr, col, d == 0 ? val : fv_mul(val, pre[(d - 1) * 32 + lane]),
                     act);
        }
      }
    }
    __syncwarp();
    chunk_id = claims ? __shfl_sync(~0u, claim, 0) : a.nchunks;
  }
}

// ---------------------------------------------------------------------------
// Scatter (S == d): every unit adds src(u) * P_{d-1} to output row
// fids[d][u], with P_{d-1} = Q * U_{d-1}[parent] and Q the prefix of the
// levels above the parent (it changes only where a unit closes two or more
// levels). Units are independent, so a warp takes 32 / W of them per step:
// W lanes per unit, 4 columns (one float4) per lane, vector atomics.
// Skewed modes send many units of a batch to the same output row, and the
// vector atomics on that row serialise; so a batch whose units repeat an
// output row first stages every unit's row in shared memory and lets the
// first unit of each repeated row add the group's sum with one atomic.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float4 lds4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ void sts4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }

// Per-warp shared memory, sized by the row width: prefix rows (kMaxModes x
// ldr), the batch's (id, value) pairs, parent ids, output-row groups and
// leaders, then the staged unit rows (kBatch x ldr).
__host__ __device__ constexpr size_t scatter_warp_bytes(int ldr) {
  return ((size_t)kMaxModes * ldr * sizeof(float) + kBatch * (sizeof(uint2) + 3 * sizeof(uint32_t)) +
          (size_t)kBatch * ldr * sizeof(float) + 15) / 16 * 16;
}

template <FactorType FT>
__device__ __forceinline__ float4 ld_factor4(const void *U, uint32_t row, int ldr, int col, bool act) {
  const fv<4> r = ld_factor<4, FT>(U, row, ldr, col, act);
  return make_float4(r.x[0], r.x[1], r.x[2], r.x[3]);
}

// Prefix rows (per column, all ldr columns; rows ldr floats apart) of levels
// lo..hi-1.
template <FactorType FT>
__device__ __noinline__ void scatter_prefix(const WalkArgs &a, float *preq, uint32_t nodeL, int lo,
                                            int hi, int lane) {
  const int c = 4 * lane;
  const bool act = c < a.ldr;
  for (int l = lo; l < hi; ++l) {
    const uint32_t n = __shfl_sync(~0u, nodeL, l);
    const bool valid = (uint64_t)n < a.nfibs[l];
    const uint32_t f = valid ? __ldg(a.fids[l] + n) : 0u;
    float4 row = ld_factor4<FT>(a.U[l], f, a.ldr, c, act && valid);
    if (l > 0 && act) {
      const float4 p = *reinterpret_cast<const float4 *>(preq + (l - 1) * a.ldr + c);
      row = make_float4(row.x * p.x, row.y * p.y, row.z * p.z, row.w * p.w);
    }
    if (act) *reinterpret_cast<float4 *>(preq + l * a.ldr + c) = row;
  }
}

template <int W, FactorType FT, bool LEAF, bool HOT>
__global__ void __launch_bounds__(256, HOT ? 3 : 1) k_scatter(const __grid_constant__ WalkArgs a) {
  constexpr int UPS = 32 / W;  // units per step
  extern __shared__ __align__(16) unsigned char walk_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char *wbase = walk_raw + (size_t)warp * scatter_warp_bytes(a.ldr);
  float *preq = reinterpret_cast<float *>(wbase);  // kMaxModes x ldr columns
  uint2 *ustage = reinterpret_cast<uint2 *>(preq + kMaxModes * a.ldr);
  uint32_t *pstage = reinterpret_cast<uint32_t *>(ustage + kBatch);
  uint32_t *gstage = pstage + kBatch;  // lanes sharing each unit's output row
  uint32_t *lstage = gstage + kBatch;  // units that lead a repeated row
  float *xs = reinterpret_cast<float *>(lstage + kBatch);  // staged unit rows
  const int slot = lane / W;
  const int col = 4 * (lane % W);
  const bool act = col < a.R;
  const int d = a.S;
  // hot output rows: summed by the block in shared memory, added to the
  // output once at the end (their atomics would otherwise queue on a few L2
  // lines); the grid is then resident and warps stride over the chunks
  double *hacc = HOT ? reinterpret_cast<double *>(walk_raw + kWarps * scatter_warp_bytes(a.ldr)) : nullptr;
  if constexpr (HOT) {
    for (int i = threadIdx.x; i < a.nhot * a.ldr; i += blockDim.x) hacc[i] = 0.0;
    __syncthreads();
  }
  auto emit = [&](uint32_t row, const float4 &x) {
    if constexpr (HOT) {
      const uint32_t sl = __ldg(a.hot_slot + row);
      if (sl != 0xFFu) {
        double *h = hacc + sl * a.ldr + col;
        atomicAdd(h, (double)x.x);
        atomicAdd(h + 1, (double)x.y);
        atomicAdd(h + 2, (double)x.z);
        atomicAdd(h + 3, (double)x.w);
        return;
      }
    }
    double *o = a.out + (size_t)row * a.ldr + col;
    atomicAdd(o, (double)x.x);
    atomicAdd(o + 1, (double)x.y);
    atomicAdd(o + 2, (double)x.z);
    atomicAdd(o + 3, (double)x.w);
  };
  // without hot rows the grid covers every chunk: one chunk per warp
  for (uint32_t chunk_id = blockIdx.x * kWarps + warp; chunk_id < a.nchunks;
       chunk_id = HOT ? chunk_id + gridDim.x * kWarps : a.nchunks) {
    const uint32_t *sc = a.sched + (size_t)chunk_id * (d + 1);
    uint32_t nodeL = lane < d ? sc[lane] : 0u;
    if (d >= 2) scatter_prefix<FT>(a, preq, nodeL, 0, d - 1, lane);
    __syncwarp();
    const uint64_t u0 = (uint64_t)chunk_id * a.chunk;
    const uint64_t u1 = min(u0 + a.chunk, a.nunits);
    for (uint64_t base = u0; base < u1; base += kBatch) {
      const int cnt = (int)min((uint64_t)kBatch, u1 - base);
      const bool in = lane < cnt;
      const uint32_t id = in ? __ldg(a.src_ids + base + lane) : 0u;
      float v = 0.f;
      if constexpr (LEAF) v = in ? __ldg(a.vals + base + lane) : 0.f;
      const uint32_t cd = (in && d >= 1) ? (uint32_t)__ldg(a.src_cd + base + lane) : 0u;
      const uint32_t M = __ballot_sync(~0u, cd >= 1u);
      const uint32_t M2 = __ballot_sync(~0u, cd >= 2u);
      // factor-row ids of the parents (level d-1) of this batch's units
      const uint32_t nodeP = d >= 1 ? __shfl_sync(~0u, nodeL, d - 1) : 0u;
      uint32_t pf = 0;
      if (d >= 1 && (uint64_t)nodeP + lane < a.nfibs[d - 1]) pf = __ldg(a.fids[d - 1] + nodeP + lane);
      ustage[lane] = make_uint2(id, __float_as_uint(v));
      pstage[lane] = pf;
      // units of this batch that repeat an output row
      const uint32_t grp = __match_any_sync(~0u, in ? id : 0xFFFFFFFFu);
      const bool lead = in && (grp & lanemask_lt()) == 0;
      const bool stage = __ballot_sync(~0u, in && !lead) != 0u;
      gstage[lane] = grp;
      __syncwarp();
      int k = 0;
      while (k < cnt) {
        const uint32_t rest = M2 & (~0u << k);
        const int deep = rest ? __ffs(rest) - 1 : 32;
        const int ke = min(deep, cnt - 1);
        float4 Q = make_float4(1.f, 1.f, 1.f, 1.f);
        if (d >= 2 && act) Q = *reinterpret_cast<const float4 *>(preq + (d - 2) * a.ldr + col);
        // four steps' row loads are issued before any of their products
        constexpr int ST = 4;
        for (int k0 = k; k0 <= ke; k0 += ST * UPS) {
          float4 r[ST];
          fv<4> m[LEAF ? 1 : ST];
#pragma unroll
          for (int t = 0; t < ST; ++t) {
            const int unit = k0 + t * UPS + slot;
            const bool ok = unit <= ke && act;
            r[t] = make_float4(1.f, 1.f, 1.f, 1.f);
            if (d >= 1) r[t] = ld_factor4<FT>(a.U[d - 1], pstage[__popc(M & ((1u << (unit & 31)) - 1u))],
                                              a.ldr, col, ok);
            if constexpr (!LEAF) m[t] = ld_rows<4>(a.src_rows, base + (unit & 31), a.ldr, col, ok);
          }
#pragma unroll
          for (int t = 0; t < ST; ++t) {
            const int unit = k0 + t * UPS + slot;
            const bool ok = unit <= ke && act;
            const uint2 e = ustage[unit & 31];
            const float4 p = d >= 1 ? make_float4(Q.x * r[t].x, Q.y * r[t].y, Q.z * r[t].z, Q.w * r[t].w)
                                    : r[t];
            float4 x;
            if constexpr (LEAF) {
              const float sv = __uint_as_float(e.y);
              x = make_float4(sv * p.x, sv * p.y, sv * p.z, sv * p.w);
            } else {
              x = make_float4(m[t].x[0] * p.x, m[t].x[1] * p.y, m[t].x[2] * p.z, m[t].x[3] * p.w);
            }
            if (ok) {
              if (stage) sts4(xs + (unit & 31) * a.ldr + col, x);
              else emit(e.x, x);
            }
          }
        }
        if (deep == ke) {
          // unit ke closes levels d-1 .. d-c (c >= 2): the levels above its
          // parent move on and Q is recomputed
          const int c = (int)__shfl_sync(~0u, cd, ke);
          if (lane >= d - c && lane < d - 1) nodeL += 1;
          if ((uint64_t)__shfl_sync(~0u, nodeL, d - c) < a.nfibs[d - c])
            scatter_prefix<FT>(a, preq, nodeL, d - c, d - 1, lane);
          __syncwarp();
        }
        k = ke + 1;
      }
      if (stage) {
        // one atomic per distinct output row: the leading unit sums its group
        __syncwarp();
        const uint32_t L = __ballot_sync(~0u, lead);
        if (lead) lstage[__popc(L & lanemask_lt())] = (uint32_t)lane;
        __syncwarp();
        const int nl = __popc(L);
        for (int i0 = 0; i0 < nl; i0 += UPS) {
          const int i = i0 + slot;
          if (i < nl && act) {
            const uint32_t u = lstage[i];
            uint32_t members = gstage[u];
            float4 sum = make_float4(0.f, 0.f, 0.f, 0.f);
            while (members) {
              const int m = __ffs(members) - 1;
              members &= members - 1u;
              const float4 x = lds4(xs + m * a.ldr + col);
              sum = make_float4(sum.x + x.x, sum.y + x.y, sum.z + x.z, sum.w + x.w);
            }
            emit(ustage[u].x, sum);
          }
        }
      }
      if (d >= 1 && lane == d - 1) nodeL += (uint32_t)__popc(M);
      __syncwarp();
    }
  }
  if constexpr (HOT) {
    __syncthreads();
    for (int i = threadIdx.x; i < a.nhot * a.ldr; i += blockDim.x) {
      const double v = hacc[i];
      if (v != 0.0) atomicAdd(a.out + (size_t)a.hot_rows[i / a.ldr] * a.ldr + i % a.ldr, v);
    }
  }
}

// Units per output row of a scatter walk (the ids of its level).
__global__ void k_row_count(const uint32_t *ids, uint64_t n, uint32_t rows, uint32_t *count) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t r = ids[i];
    if (r < rows) atomicAdd(count + r, 1u);
  }
}

// Schedule: for chunk c, the node of every level 0..S-1 that contains the
// chunk's first unit, and which of those nodes started before it.
__global__ void k_schedule(WalkArgs a, uint32_t *sched) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.nchunks) return;
  const int S = a.S;
  const uint64_t u0 = (uint64_t)c * a.chunk;
  uint32_t child = (uint32_t)u0;
  uint32_t mask = 0;
  bool below_partial = false;
  for (int l = S - 1; l >= 0; --l) {
    // largest n with fptr[l][n] <= child
    const uint32_t *fp = a.fptr[l];
    uint64_t lo = 0, hi = a.nfibs[l] - 1;
    while (lo < hi) {
      const uint64_t mid = (lo + hi + 1) >> 1;
      if (fp[mid] <= child)
        lo = mid;
      else
        hi = mid - 1;
    }
    const uint32_t n = (uint32_t)lo;
    const bool p = (fp[n] < child) || below_partial;
    if (p) mask |= 1u << l;
    below_partial = p;
    sched[(size_t)c * (S + 1) + l] = n;
    child = n;
  }
  sched[(size_t)c * (S + 1) + S] = mask;
}

// ---------------------------------------------------------------------------
// Deterministic accumulation: chain sums of cut nodes, prefix rows, pulls.
// ---------------------------------------------------------------------------
constexpr uint32_t kChainGroup = 32;  // partials one warp sums per group
constexpr uint32_t kPullSeg = 256;    // units per pull segment (whole rows) and per piece, at most

struct ChainArgs {
  const float *span;
  int span_nlev, ldr, R;
  int span_lev[kMaxModes];
  const uint32_t *chains;  // 6 per chain
  const uint32_t *groups;  // 3 per group
  uint32_t nchains, ngroups;
  double *gsum;
  float *store[kMaxModes];
  double *out;             // level-0 output rows (output level 0), else nullptr
  const uint32_t *root_ids;
};

// Partial k of the chain of a node cut by the boundaries of chunks
// c_first..c_last: k <= c_last - c_first is the tail of chunk c_first-1+k,
// the last one the head of chunk c_last (where the node closes).
__device__ __forceinline__ const float *chain_partial(const ChainArgs &a, int ls, uint32_t c_first,
                                                      uint32_t c_last, uint32_t k) {
  const uint32_t ntail = c_last - c_first + 1;
  const uint32_t c = k < ntail ? c_first - 1 + k : c_last;
  const int which = k < ntail ? 1 : 0;
  return a.span + (((size_t)c * a.span_nlev + ls) * 2 + which) * a.ldr;
}

// One warp per group: its partials summed in chunk order.
__global__ void k_chain_groups(const __grid_constant__ ChainArgs a) {
  const uint32_t g = (uint32_t)((blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (g >= a.ngroups) return;
  const uint32_t ch = a.groups[3 * (size_t)g], k0 = a.groups[3 * (size_t)g + 1],
                 cnt = a.groups[3 * (size_t)g + 2];
  const uint32_t *c = a.chains + 6 * (size_t)ch;
  const int ls = a.span_lev[c[0]];
  for (int col = lane; col < a.R; col += 32) {
    // loads issued eight at a time, added in chunk order
    double acc = 0.0;
    uint32_t k = k0;
    for (; k + 8 <= k0 + cnt; k += 8) {
      float v[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) v[q] = chain_partial(a, ls, c[2], c[3], k + q)[col];
#pragma unroll
      for (int q = 0; q < 8; ++q) acc += (double)v[q];
    }
    for (; k < k0 + cnt; ++k) acc += (double)chain_partial(a, ls, c[2], c[3], k)[col];
    a.gsum[(size_t)g * a.ldr + col] = acc;
  }
}

// Sum of n FP64 rows (stride ldr) in index order, column col: loads issued
// eight at a time.
__device__ __forceinline__ double ordered_sum(const double *rows, uint64_t n, int ldr, int col) {
  double acc = 0.0;
  uint64_t k = 0;
  for (; k + 8 <= n; k += 8) {
    double v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = rows[(k + q) * ldr + col];
#pragma unroll
    for (int q = 0; q < 8; ++q) acc += v[q];
  }
  for (; k < n; ++k) acc += rows[k * ldr + col];
  return acc;
}

// Sum of n FP64 rows in index order by a whole block: warp w sums the w-th
// of 8 contiguous ranges, then the 8 range sums are added in order. The
// split depends only on n, so the result does not depend on scheduling.
__device__ __forceinline__ void block_ordered_sum(const double *rows, uint64_t n, int ldr, int R,
                                                  double *red /* kWarps x R */, double *out_col) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t per = (n + kWarps - 1) / kWarps;
  const uint64_t b = min(n, (uint64_t)warp * per), e = min(n, b + per);
  for (int col = lane; col < R; col += 32)
    red[warp * R + col] = ordered_sum(rows + b * ldr, e - b, ldr, col);
  __syncthreads();
  if (warp == 0)
    for (int col = lane; col < R; col += 32) {
      double acc = 0.0;
      for (int w = 0; w < kWarps; ++w) acc += red[w * R + col];
      out_col[col] = acc;
    }
  __syncthreads();
}

// A chain's total, stored to the node's memo row and, at level 0 with a
// root output, to its output row.
__device__ __forceinline__ void chain_store(const ChainArgs &a, const uint32_t *c, int col, double v) {
  const int l = (int)c[0];
  const uint32_t node = c[1];
  if (a.store[l]) a.store[l][(size_t)node * a.ldr + col] = (float)v;
  if (l == 0 && a.out) a.out[(size_t)a.root_ids[node] * a.ldr + col] = v;
}

// Chains of at most kChainShort groups: one warp each, the group sums in
// order.
constexpr uint32_t kChainShort = 16;
__global__ void k_chain_finish(const __grid_constant__ ChainArgs a, const uint32_t *ids, uint32_t n) {
  const uint32_t i = (uint32_t)((blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  const uint32_t *c = a.chains + 6 * (size_t)ids[i];
  for (int col = lane; col < a.R; col += 32)
    chain_store(a, c, col, ordered_sum(a.gsum + (size_t)c[4] * a.ldr, c[5], a.ldr, col));
}

// Longer chains (a skewed root slice cut by thousands of chunks): one block
// each.
__global__ void __launch_bounds__(256) k_chain_finish_long(const __grid_constant__ ChainArgs a,
                                                           const uint32_t *ids) {
  __shared__ double red[kWarps * 128];
  __shared__ double tot[128];
  const uint32_t *c = a.chains + 6 * (size_t)ids[blockIdx.x];
  block_ordered_sum(a.gsum + (size_t)c[4] * a.ldr, c[5], a.ldr, a.R, red, tot);
  for (int col = threadIdx.x; col < a.R; col += blockDim.x) chain_store(a, c, col, tot[col]);
}

// parent[c] = p for the children c of every node p (fptr of the parent level).
__global__ void k_fill_parent(const uint32_t *fptr, uint64_t nparent, uint32_t *parent) {
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < nparent;
       p += (uint64_t)gridDim.x * blockDim.x)
    for (uint32_t c = fptr[p]; c < fptr[p + 1]; ++c) parent[c] = (uint32_t)p;
}

// Prefix rows of one level: P_l[n] = P_{l-1}[parent(n)] * U_l[fids_l[n]]
// (P_0[n] = U_0[fids_0[n]]); padding columns are zero.
template <FactorType FT>
__global__ void k_prefix_level(const void *U, const uint32_t *fids, const uint32_t *parent,
                               const float *prev, uint64_t n, int R, int ldr, float *out) {
  const int q = ldr / 4;
  const uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (e >= n * (uint64_t)q) return;
  const uint64_t node = e / q;
  const int col = 4 * (int)(e % q);
  const fv<4> u = ld_factor<4, FT>(U, fids[node], ldr, col, col < R);
  float4 r = make_float4(u.x[0], u.x[1], u.x[2], u.x[3]);
  if (prev) {
    const float4 p = *reinterpret_cast<const float4 *>(prev + (size_t)parent[node] * ldr + col);
    r = make_float4(r.x * p.x, r.y * p.y, r.z * p.z, r.w * p.w);
  }
  *reinterpret_cast<float4 *>(out + node * ldr + col) = r;
}

struct PullArgs {
  int d, R, ldr;
  const uint32_t *perm, *prow, *pparent, *segs;
  uint32_t nsegs;
  const float *vals;      // leaf values (leaf source)
  const float *src_rows;  // node rows of level d (row source)
  const float *prefix;    // P_{d-1} rows (d >= 1)
  double *out;
  double *piece_sum;
};

// Pull scatter: one warp per segment of units sorted by output row; each
// unit's contribution src(u) * P_{d-1}[parent(u)] is added in that order and
// a row is stored once, when its last unit is done (whole rows), or into its
// piece's slot (long rows, summed in order by k_piece_sum).
template <int V, bool LEAF>
__global__ void __launch_bounds__(256) k_pull(const __grid_constant__ PullArgs a) {
  __shared__ uint4 stage[kWarps][kBatch];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int col = lane * V;
  const bool act = col < a.R;
  constexpr int SB = 8;
  for (uint32_t sg = blockIdx.x * kWarps + warp; sg < a.nsegs; sg += gridDim.x * kWarps) {
    const uint32_t jb = a.segs[3 * (size_t)sg], je = a.segs[3 * (size_t)sg + 1],
                   slot = a.segs[3 * (size_t)sg + 2];
    double acc[V];
#pragma unroll
    for (int i = 0; i < V; ++i) acc[i] = 0.0;
    uint32_t cur = a.prow[jb];
    auto flush = [&](uint32_t row) {
      if (!act) return;
      double *p = (slot == 0xFFFFFFFFu ? a.out + (size_t)row * a.ldr : a.piece_sum + (size_t)slot * a.ldr) + col;
#pragma unroll
      for (int i = 0; i < V; ++i) p[i] = acc[i];
    };
    for (uint32_t j0 = jb; j0 < je; j0 += kBatch) {
      const int cnt = (int)min((uint32_t)kBatch, je - j0);
      if (lane < cnt) {
        const uint32_t u = a.perm[j0 + lane];
        const float v = LEAF ? a.vals[u] : 0.f;
        stage[warp][lane] = make_uint4(u, a.prow[j0 + lane], a.d >= 1 ? a.pparent[j0 + lane] : 0u,
                                       __float_as_uint(v));
      }
      __syncwarp();
      for (int k0 = 0; k0 < cnt; k0 += SB) {
        fv<V> x[SB];
#pragma unroll
        for (int q = 0; q < SB; ++q) {
          const int k = k0 + q;
          const bool ok = k < cnt;
          const uint4 e = stage[warp][ok ? k : 0];
          fv<V> t;
          if constexpr (LEAF) t = fv_fill<V>(__uint_as_float(e.w));
          else t = ld_rows<V>(a.src_rows, e.x, a.ldr, col, ok && act);
          if (a.d >= 1) t = fv_mul(t, ld_rows<V>(a.prefix, e.z, a.ldr, col, ok && act));
          x[q] = t;
        }
#pragma unroll
        for (int q = 0; q < SB; ++q) {
          const int k = k0 + q;
          if (k < cnt) {
            const uint32_t row = stage[warp][k].y;
            if (row != cur) {
              flush(cur);
#pragma unroll
              for (int i = 0; i < V; ++i) acc[i] = 0.0;
              cur = row;
            }
#pragma unroll
            for (int i = 0; i < V; ++i) acc[i] += (double)x[q].x[i];
          }
        }
      }
      __syncwarp();
    }
    flush(cur);
  }
}

// One block per long row: its pieces summed in order.
__global__ void __launch_bounds__(256) k_piece_sum(const uint32_t *pieces, const double *piece_sum,
                                                   int R, int ldr, double *out) {
  __shared__ double red[kWarps * 128];
  __shared__ double tot[128];
  const uint32_t i = blockIdx.x;
  const uint32_t row = pieces[3 * (size_t)i], p0 = pieces[3 * (size_t)i + 1],
                 np = pieces[3 * (size_t)i + 2];
  block_ordered_sum(piece_sum + (size_t)p0 * ldr, np, ldr, R, red, tot);
  for (int col = threadIdx.x; col < R; col += blockDim.x) out[(size_t)row * ldr + col] = tot[col];
}

WalkArgs make_args(const TreeWalk &w, const LevelFactors *f, double *out) {
  WalkArgs a;
  const DevCsf &c = *w.csf;
  a.N = w.nmodes;
  a.S = w.src;
  a.d = w.out;
  a.R = w.R;
  a.ldr = w.ldr;
  a.chunk = w.chunk;
  a.nchunks = w.nchunks;
  a.nunits = w.nunits;
  for (int l = 0; l < kMaxModes; ++l) {
    a.nfibs[l] = c.nfibs[l];
    a.fptr[l] = c.fptr[l].get();
    a.fids[l] = c.fids[l].get();
    a.U[l] = f ? f->U[l] : nullptr;
    a.store[l] = w.store[l];
  }
  a.vals = c.vals32.get();
  a.src_rows = w.src_rows;
  a.src_ids = c.fids[w.src].get();
  a.src_cd = w.src >= 1 ? c.cdepth[w.src].get() : nullptr;
  a.U_src = f ? f->U[w.src] : nullptr;
  a.out = out;
  a.sched = w.sched.get();
  a.counter = w.sched.get() ? w.sched.get() + (size_t)w.nchunks * (w.src + 1) : nullptr;
  a.nhot = w.nhot;
  a.hot_slot = w.hot_slot.get();
  a.hot_rows = w.hot_rows.get();
  a.span = w.span_nlev > 0 ? w.span.get() : nullptr;
  a.span_nlev = w.span_nlev;
  for (int l = 0; l < kMaxModes; ++l) a.span_lev[l] = w.span_lev[l];
  return a;
}

// Blocks of `kernel` that fit on the device at once with `smem` bytes each.
template <typename K>
unsigned resident_blocks(K kernel, int threads, size_t smem) {
  int dev = 0, sms = 0, per_sm = 0;
  ADATM_CUDA(cudaGetDevice(&dev));
  ADATM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  ADATM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
  return (unsigned)std::max(1, sms * std::max(1, per_sm));
}

template <int V, int W, int VW, FactorType FT, bool LEAF, int F>
void launch_contract_v(const WalkArgs &a, unsigned blocks, bool resident, cudaStream_t s) {
  const size_t smem = contract_smem<V>(a.N);
  auto kern = k_contract<V, W, VW, FT, LEAF, F>;
  if (resident) {
    blocks = std::min(blocks, resident_blocks(kern, 256, smem));
    ADATM_CUDA(cudaMemsetAsync(a.counter, 0, sizeof(uint32_t), s));
    kern<<<blocks, 256, smem, s>>>(a);
  } else {
    WalkArgs b = a;
    b.counter = nullptr;  // one chunk per warp: blocks cover every chunk
    kern<<<blocks, 256, smem, s>>>(b);
  }
}

// Levels folded into the source loop: level S-1 whenever it is neither
// stored nor the output level (a level-(S-1) item costs more than the extra
// gather per unit at any fan-out the trees show); level S-2 as well when it
// too is unstored and above d and holds at most kFold2Units source units per
// node on average (at higher fan-out the extra gather per unit costs more
// than the items it saves). `want` >= 0 caps the count.
constexpr double kFold2Units = 4.0;
int fold_levels(const WalkArgs &a, int want) {
  const int cap = want < 0 ? 2 : std::min(want, 2);
  int f = 0;
  while (f < cap && a.S - 1 - f > a.d && a.store[a.S - 1 - f] == nullptr) ++f;
  if (want < 0 && f == 2 && (double)a.nunits > kFold2Units * (double)a.nfibs[a.S - 2]) f = 1;
  return f;
}

// The (V, W, VW) shapes the contraction is built for: V columns per lane in
// the level loop (32 lanes cover the rank), W walkers in the source loop
// with VW columns per lane (32 / W lanes cover the rank).
#define ADATM_CONTRACT_SHAPES(X) \
  X(1, 1, 1) X(1, 2, 1) X(1, 2, 2) X(1, 4, 1) X(1, 4, 2) X(1, 4, 4) X(2, 1, 2) X(2, 2, 4) X(4, 1, 4)

// Columns per walker lane for W walkers at rank R (0 if W walkers cannot
// cover R with at most 4 columns per lane).
int walker_cols(int R, int W) {
  for (int vw : {1, 2, 4})
    if ((32 / W) * vw >= R) return vw;
  return 0;
}

template <FactorType FT, bool LEAF>
void launch_contract(int vec, int walkers, int fold, const WalkArgs &a, unsigned blocks, bool resident,
                     cudaStream_t s) {
  const int f = fold_levels(a, fold);
  const int vw = walker_cols(a.R, walkers);
#define ADATM_CONTRACT_CASE(V, W, VW)                                                  \
  if (vec == V && walkers == W && vw == VW) {                                          \
    if (f == 2) launch_contract_v<V, W, VW, FT, LEAF, 2>(a, blocks, resident, s);      \
    else if (f == 1) launch_contract_v<V, W, VW, FT, LEAF, 1>(a, blocks, resident, s); \
    else launch_contract_v<V, W, VW, FT, LEAF, 0>(a, blocks, resident, s);             \
    ADATM_LAUNCH();                                                                    \
    return;                                                                            \
  }
  ADATM_CONTRACT_SHAPES(ADATM_CONTRACT_CASE)
#undef ADATM_CONTRACT_CASE
  throw BadInput("no contraction kernel for " + std::to_string(walkers) + " walkers at rank " +
                 std::to_string(a.R));
}

template <int W, FactorType FT, bool LEAF>
void launch_scatter_w(const WalkArgs &a, unsigned blocks, cudaStream_t s) {
  if (a.nhot > 0) {
    // each block sums the hot rows once: as few blocks as fit at once
    const size_t smem = kWarps * scatter_warp_bytes(a.ldr) + (size_t)a.nhot * a.ldr * sizeof(double);
    blocks = std::min(blocks, resident_blocks(k_scatter<W, FT, LEAF, true>, 256, smem));
    k_scatter<W, FT, LEAF, true><<<blocks, 256, smem, s>>>(a);
  } else {
    k_scatter<W, FT, LEAF, false><<<blocks, 256, kWarps * scatter_warp_bytes(a.ldr), s>>>(a);
  }
}

template <FactorType FT, bool LEAF>
void launch_scatter(int w, const WalkArgs &a, unsigned blocks, cudaStream_t s) {
  switch (w) {
    case 4: launch_scatter_w<4, FT, LEAF>(a, blocks, s); break;
    case 8: launch_scatter_w<8, FT, LEAF>(a, blocks, s); break;
    case 16: launch_scatter_w<16, FT, LEAF>(a, blocks, s); break;
    case 32: launch_scatter_w<32, FT, LEAF>(a, blocks, s); break;
    default: throw BadInput("unsupported lanes per unit");
  }
  ADATM_LAUNCH();
}

// Contraction: columns per lane (32 lanes cover R).
int vec_for_rank(int R) {
  if (R <= 32) return 1;
  if (R <= 64) return 2;
  if (R <= 128) return 4;
  throw BadInput("rank above 128 is not supported by the GPU kernels");
}

}  // namespace

int default_walkers(int R) { return R <= 64 ? 2 : 1; }

bool walkers_supported(int R, int W) {
  if (W != 1 && W != 2 && W != 4) return false;
  const int v = R <= 32 ? 1 : (R <= 64 ? 2 : 4);
  const int vw = walker_cols(R, W);
  if (vw == 0) return false;
#define ADATM_CONTRACT_OK(V, WW, VW) \
  if (v == V && W == WW && vw == VW) return true;
  ADATM_CONTRACT_SHAPES(ADATM_CONTRACT_OK)
#undef ADATM_CONTRACT_OK
  return false;
}

namespace {

// Scatter: lanes per unit (4 columns per lane).
int lanes_for_rank(int R) {
  if (R <= 16) return 4;
  if (R <= 32) return 8;
  if (R <= 64) return 16;
  if (R <= 128) return 32;
  throw BadInput("rank above 128 is not supported by the GPU kernels");
}

}  // namespace

void set_walk_attributes() {
  static bool done = false;
  if (done) return;
#define ADATM_ATTR_C0(V, W, VW, FT, LEAF, F)                                      \
  ADATM_CUDA(cudaFuncSetAttribute(k_contract<V, W, VW, FT, LEAF, F>,              \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                                  (int)contract_smem<V>(kMaxModes)));
#define ADATM_ATTR_C1(V, W, VW, FT, LEAF) \
  ADATM_ATTR_C0(V, W, VW, FT, LEAF, 0)    \
  ADATM_ATTR_C0(V, W, VW, FT, LEAF, 1)    \
  ADATM_ATTR_C0(V, W, VW, FT, LEAF, 2)
#define ADATM_ATTR_CS(V, W, VW)                       \
  ADATM_ATTR_C1(V, W, VW, FactorType::F32, true)      \
  ADATM_ATTR_C1(V, W, VW, FactorType::F32, false)     \
  ADATM_ATTR_C1(V, W, VW, FactorType::BF16, true)     \
  ADATM_ATTR_C1(V, W, VW, FactorType::BF16, false)
#define ADATM_ATTR_S(W, FT, LEAF)                                                 \
  ADATM_CUDA(cudaFuncSetAttribute(k_scatter<W, FT, LEAF, false>,                  \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                                  (int)(kWarps * scatter_warp_bytes(128))));      \
  ADATM_CUDA(cudaFuncSetAttribute(k_scatter<W, FT, LEAF, true>,                   \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                                  (int)(kWarps * scatter_warp_bytes(128) +        \
                                        kHotRows * 128 * sizeof(double))));
#define ADATM_ATTR_ALL(M, X)                \
  M(X, FactorType::F32, true)               \
  M(X, FactorType::F32, false)              \
  M(X, FactorType::BF16, true)              \
  M(X, FactorType::BF16, false)
  ADATM_CONTRACT_SHAPES(ADATM_ATTR_CS)
  ADATM_ATTR_ALL(ADATM_ATTR_S, 4)
  ADATM_ATTR_ALL(ADATM_ATTR_S, 8)
  ADATM_ATTR_ALL(ADATM_ATTR_S, 16)
  ADATM_ATTR_ALL(ADATM_ATTR_S, 32)
#undef ADATM_ATTR_ALL
#undef ADATM_ATTR_S
#undef ADATM_ATTR_CS
#undef ADATM_ATTR_C1
#undef ADATM_ATTR_C0
  done = true;
}

// ---------------------------------------------------------------------------
// Deterministic walks: preparation and launch.
// ---------------------------------------------------------------------------
namespace {

template <typename T>
std::vector<T> to_host(const T *dev, size_t n, cudaStream_t s) {
  std::vector<T> h(n);
  if (n) ADATM_CUDA(cudaMemcpyAsync(h.data(), dev, n * sizeof(T), cudaMemcpyDeviceToHost, s));
  ADATM_CUDA(cudaStreamSynchronize(s));
  return h;
}

template <typename T>
void to_device(DevBuf<T> &dst, const std::vector<T> &h, cudaStream_t s) {
  dst.alloc(std::max<size_t>(h.size(), 1));
  if (!h.empty())
    ADATM_CUDA(cudaMemcpyAsync(dst.get(), h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  ADATM_CUDA(cudaStreamSynchronize(s));
}

// Slots and chains of a contraction: levels whose cut nodes would otherwise
// take atomics (stored levels, and level 0 when it is the output), and for
// each node a chunk boundary cuts, the run of chunks it spans. Deterministic
// contractions below the root also store their level-d sums for the pull.
void prepare_spans(TreeWalk &w, cudaStream_t s) {
  const DevCsf &c = *w.csf;
  const int S = w.src, d = w.out;
  if (w.deterministic && d > 0) {
    // the level-d sums are stored, then pulled into the output rows
    w.level_rows.alloc((size_t)std::max<uint64_t>(c.nfibs[d], 1) * w.ldr);
    ADATM_CUDA(cudaMemsetAsync(w.level_rows.get(), 0, w.level_rows.bytes(), s));
    w.store[d] = w.level_rows.get();
    w.pull = true;
  }
  w.span_nlev = 0;
  for (int l = 0; l < kMaxModes; ++l) w.span_lev[l] = -1;
  for (int l = 0; l < S; ++l)
    if (w.store[l] != nullptr || (l == 0 && d == 0)) w.span_lev[l] = w.span_nlev++;
  w.nchains = w.ngroups = 0;
  if (w.nchunks == 0 || w.span_nlev == 0) return;
  w.span.alloc((size_t)w.nchunks * w.span_nlev * 2 * w.ldr);
  const std::vector<uint32_t> sc = to_host(w.sched.get(), (size_t)w.nchunks * (S + 1), s);
  std::vector<uint32_t> chains, groups;
  const size_t st = (size_t)S + 1;
  for (int l = 0; l < S; ++l) {
    if (w.span_lev[l] < 0) continue;
    uint32_t ch = 1;
    while (ch < w.nchunks) {
      if (!((sc[ch * st + S] >> l) & 1u)) {
        ++ch;
        continue;
      }
      const uint32_t node = sc[ch * st + l];
      uint32_t last = ch;
      while (last + 1 < w.nchunks && ((sc[(last + 1) * st + S] >> l) & 1u) &&
             sc[(last + 1) * st + l] == node)
        ++last;
      const uint32_t npart = (last - ch + 1) + 1;
      const uint32_t id = (uint32_t)(chains.size() / 6);
      const uint32_t g0 = (uint32_t)(groups.size() / 3);
      const uint32_t ng = (npart + kChainGroup - 1) / kChainGroup;
      for (uint32_t k0 = 0; k0 < npart; k0 += kChainGroup) {
        groups.push_back(id);
        groups.push_back(k0);
        groups.push_back(std::min(kChainGroup, npart - k0));
      }
      const uint32_t row[6] = {(uint32_t)l, node, ch, last, g0, ng};
      chains.insert(chains.end(), row, row + 6);
      ch = last + 1;
    }
  }
  w.nchains = (uint32_t)(chains.size() / 6);
  w.ngroups = (uint32_t)(groups.size() / 3);
  // short chains first (a warp each), then long ones (a block each)
  std::vector<uint32_t> ids;
  for (uint32_t i = 0; i < w.nchains; ++i)
    if (chains[6 * (size_t)i + 5] <= kChainShort) ids.push_back(i);
  w.nshort = (uint32_t)ids.size();
  for (uint32_t i = 0; i < w.nchains; ++i)
    if (chains[6 * (size_t)i + 5] > kChainShort) ids.push_back(i);
  to_device(w.chain_ids, ids, s);
  to_device(w.chains, chains, s);
  to_device(w.groups, groups, s);
  w.gsum.alloc((size_t)std::max<uint32_t>(w.ngroups, 1) * w.ldr);
}

// The pull of level d = w.out: units (level-d nodes) in a stable order by
// output row, their parents, segments of whole rows and pieces of long rows,
// the parent arrays and prefix buffers of the levels above.
void det_prepare_pull(TreeWalk &w, cudaStream_t s) {
  const DevCsf &c = *w.csf;
  const int d = w.out;
  const uint64_t n = c.nfibs[d];
  const uint64_t rows = c.dims[c.dim_perm[d]];
  const std::vector<uint32_t> fid = to_host(c.fids[d].get(), n, s);
  std::vector<uint32_t> par;
  if (d >= 1) {
    const std::vector<uint32_t> fp = to_host(c.fptr[d - 1].get(), c.nfibs[d - 1] + 1, s);
    par.assign(n, 0);
    for (uint64_t p = 0; p < c.nfibs[d - 1]; ++p)
      for (uint32_t u = fp[p]; u < fp[p + 1] && u < n; ++u) par[u] = (uint32_t)p;
  }
  // stable counting sort by output row
  std::vector<uint64_t> start(rows + 1, 0);
  for (uint64_t u = 0; u < n; ++u) ++start[fid[u] + 1];
  for (uint64_t r = 0; r < rows; ++r) start[r + 1] += start[r];
  std::vector<uint32_t> perm(n), prow(n), pparent(d >= 1 ? n : 0);
  {
    std::vector<uint64_t> pos(start.begin(), start.end() - 1);
    for (uint64_t u = 0; u < n; ++u) {
      const uint64_t j = pos[fid[u]]++;
      perm[j] = (uint32_t)u;
      prow[j] = fid[u];
      if (d >= 1) pparent[j] = par[u];
    }
  }
  // segments: whole rows packed up to `seg` units (kPullSeg, shorter for
  // small levels so the segments still fill the device); longer rows in pieces
  uint64_t seg = kPullSeg;
  while (seg > 32 && n / seg < 148ull * 32) seg /= 2;
  std::vector<uint32_t> segs, pieces;
  uint32_t npieces = 0;
  uint64_t seg_start = 0, seg_len = 0;
  auto close_seg = [&](uint64_t end) {
    if (seg_len > 0) {
      segs.push_back((uint32_t)seg_start);
      segs.push_back((uint32_t)end);
      segs.push_back(0xFFFFFFFFu);
    }
    seg_start = end;
    seg_len = 0;
  };
  for (uint64_t r = 0; r < rows; ++r) {
    const uint64_t b = start[r], cnt = start[r + 1] - b;
    if (cnt == 0) continue;
    if (cnt > seg) {
      close_seg(b);
      const uint32_t np = (uint32_t)((cnt + seg - 1) / seg);
      pieces.push_back((uint32_t)r);
      pieces.push_back(npieces);
      pieces.push_back(np);
      for (uint32_t q = 0; q < np; ++q) {
        segs.push_back((uint32_t)(b + (uint64_t)q * seg));
        segs.push_back((uint32_t)std::min<uint64_t>(b + (uint64_t)(q + 1) * seg, b + cnt));
        segs.push_back(npieces + q);
      }
      npieces += np;
      seg_start = b + cnt;
      continue;
    }
    if (seg_len + cnt > seg) close_seg(b);
    seg_len += cnt;
  }
  close_seg(n);
  w.nsegs = (uint32_t)(segs.size() / 3);
  w.nlong = (uint32_t)(pieces.size() / 3);
  w.npieces = npieces;
  to_device(w.perm, perm, s);
  to_device(w.prow, prow, s);
  to_device(w.pparent, pparent, s);
  to_device(w.segs, segs, s);
  to_device(w.pieces, pieces, s);
  w.piece_sum.alloc((size_t)std::max<uint32_t>(npieces, 1) * w.ldr);
  // parents and prefix rows of levels 1..d-1
  uint64_t maxf = 1;
  for (int l = 0; l < d; ++l) maxf = std::max<uint64_t>(maxf, c.nfibs[l]);
  for (int l = 1; l < d; ++l) {
    w.parent[l].alloc(std::max<uint64_t>(c.nfibs[l], 1));
    const uint64_t np = c.nfibs[l - 1];
    if (np == 0) continue;
    k_fill_parent<<<(unsigned)std::min<uint64_t>((np + 255) / 256, 65535), 256, 0, s>>>(
        c.fptr[l - 1].get(), np, w.parent[l].get());
    ADATM_LAUNCH();
  }
  if (d >= 1) w.prefix[0].alloc(maxf * w.ldr);
  if (d >= 2) w.prefix[1].alloc(maxf * w.ldr);
  ADATM_CUDA(cudaStreamSynchronize(s));
}

template <FactorType FT>
void launch_prefix(const TreeWalk &w, const LevelFactors &f, cudaStream_t s) {
  const DevCsf &c = *w.csf;
  for (int l = 0; l < w.out; ++l) {
    const uint64_t n = c.nfibs[l];
    if (n == 0) continue;
    const uint64_t thr = n * (uint64_t)(w.ldr / 4);
    k_prefix_level<FT><<<(unsigned)((thr + 255) / 256), 256, 0, s>>>(
        f.U[l], c.fids[l].get(), l ? w.parent[l].get() : nullptr,
        l ? w.prefix[(l - 1) & 1].get() : nullptr, n, w.R, w.ldr, w.prefix[l & 1].get());
    ADATM_LAUNCH();
  }
}

void launch_pull(const TreeWalk &w, const LevelFactors &f, FactorType ft, const float *rows,
                 double *out, cudaStream_t s) {
  if (w.nsegs == 0) return;
  if (ft == FactorType::F32) launch_prefix<FactorType::F32>(w, f, s);
  else launch_prefix<FactorType::BF16>(w, f, s);
  PullArgs a;
  a.d = w.out;
  a.R = w.R;
  a.ldr = w.ldr;
  a.perm = w.perm.get();
  a.prow = w.prow.get();
  a.pparent = w.pparent.get();
  a.segs = w.segs.get();
  a.nsegs = w.nsegs;
  a.vals = w.csf->vals32.get();
  a.src_rows = rows;
  a.prefix = w.out >= 1 ? w.prefix[(w.out - 1) & 1].get() : nullptr;
  a.out = out;
  a.piece_sum = w.piece_sum.get();
  const bool leaf = rows == nullptr;
  const unsigned blocks = (w.nsegs + kWarps - 1) / kWarps;
  switch (vec_for_rank(w.R)) {
    case 1: leaf ? k_pull<1, true><<<blocks, 256, 0, s>>>(a) : k_pull<1, false><<<blocks, 256, 0, s>>>(a); break;
    case 2: leaf ? k_pull<2, true><<<blocks, 256, 0, s>>>(a) : k_pull<2, false><<<blocks, 256, 0, s>>>(a); break;
    default: leaf ? k_pull<4, true><<<blocks, 256, 0, s>>>(a) : k_pull<4, false><<<blocks, 256, 0, s>>>(a); break;
  }
  ADATM_LAUNCH();
  if (w.nlong) {
    k_piece_sum<<<w.nlong, 256, 0, s>>>(w.pieces.get(), w.piece_sum.get(), w.R, w.ldr, out);
    ADATM_LAUNCH();
  }
}

void launch_chains(const TreeWalk &w, double *out, cudaStream_t s) {
  if (w.nchains == 0) return;
  ChainArgs a;
  a.span = w.span.get();
  a.span_nlev = w.span_nlev;
  a.ldr = w.ldr;
  a.R = w.R;
  for (int l = 0; l < kMaxModes; ++l) {
    a.span_lev[l] = w.span_lev[l];
    a.store[l] = w.store[l];
  }
  a.chains = w.chains.get();
  a.groups = w.groups.get();
  a.nchains = w.nchains;
  a.ngroups = w.ngroups;
  a.gsum = w.gsum.get();
  a.out = w.out == 0 ? out : nullptr;
  a.root_ids = w.csf->fids[0].get();
  k_chain_groups<<<(unsigned)(((uint64_t)w.ngroups * 32 + 255) / 256), 256, 0, s>>>(a);
  ADATM_LAUNCH();
  if (w.nshort) {
    k_chain_finish<<<(unsigned)(((uint64_t)w.nshort * 32 + 255) / 256), 256, 0, s>>>(
        a, w.chain_ids.get(), w.nshort);
    ADATM_LAUNCH();
  }
  if (w.nchains > w.nshort) {
    k_chain_finish_long<<<w.nchains - w.nshort, 256, 0, s>>>(a, w.chain_ids.get() + w.nshort);
    ADATM_LAUNCH();
  }
}

}  // namespace

// The output rows of a scatter walk hit by the most units (at most
// kHotRows, each by at least kHotMin units), and the row -> slot table.
void find_hot_rows(TreeWalk &w, cudaStream_t s) {
  const DevCsf &c = *w.csf;
  const uint64_t rows64 = c.dims[c.dim_perm[w.out]];
  // a count per output row, on the device and the host: outputs with more
  // rows than kHotScanRows keep the plain scatter
  if (rows64 == 0 || rows64 > kHotScanRows) return;
  const uint32_t rows = (uint32_t)rows64;
  DevBuf<uint32_t> count(rows);
  ADATM_CUDA(cudaMemsetAsync(count.get(), 0, rows * sizeof(uint32_t), s));
  const unsigned blocks = (unsigned)std::min<uint64_t>((w.nunits + 255) / 256, 4096);
  k_row_count<<<blocks, 256, 0, s>>>(c.fids[w.out].get(), w.nunits, rows, count.get());
  ADATM_LAUNCH();
  std::vector<uint32_t> h(rows);
  ADATM_CUDA(cudaMemcpyAsync(h.data(), count.get(), rows * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  ADATM_CUDA(cudaStreamSynchronize(s));
  std::vector<uint32_t> order(rows);
  for (uint32_t r = 0; r < rows; ++r) order[r] = r;
  const uint32_t k = std::min<uint32_t>(kHotRows, rows);
  std::partial_sort(order.begin(), order.begin() + k, order.end(),
                    [&](uint32_t x, uint32_t y) { return h[x] > h[y] || (h[x] == h[y] && x < y); });
  std::vector<uint32_t> hot;
  for (uint32_t i = 0; i < k; ++i)
    if (h[order[i]] >= kHotMin) hot.push_back(order[i]);
  if (hot.empty()) return;
  std::vector<uint8_t> slot(rows, 0xFF);
  for (size_t i = 0; i < hot.size(); ++i) slot[hot[i]] = (uint8_t)i;
  w.hot_slot.alloc(rows);
  w.hot_rows.alloc(hot.size());
  ADATM_CUDA(cudaMemcpyAsync(w.hot_slot.get(), slot.data(), rows, cudaMemcpyHostToDevice, s));
  ADATM_CUDA(cudaMemcpyAsync(w.hot_rows.get(), hot.data(), hot.size() * sizeof(uint32_t),
                             cudaMemcpyHostToDevice, s));
  ADATM_CUDA(cudaStreamSynchronize(s));
  w.nhot = (int)hot.size();
}

void walk_prepare(TreeWalk &w, cudaStream_t s) {
  set_walk_attributes();
  const DevCsf &c = *w.csf;
  w.nmodes = c.nmodes;
  w.nunits = c.nfibs[w.src];
  if (w.chunk == 0) w.chunk = 32;
  w.nchunks = (uint32_t)((w.nunits + w.chunk - 1) / w.chunk);
  w.sched.alloc((size_t)std::max<uint32_t>(w.nchunks, 1) * (w.src + 1) + 1);  // + the chunk counter
  w.nhot = 0;
  w.hot_slot.reset();
  w.hot_rows.reset();
  if (w.nchunks == 0) return;
  WalkArgs a = make_args(w, nullptr, nullptr);
  k_schedule<<<(w.nchunks + 255) / 256, 256, 0, s>>>(a, w.sched.get());
  ADATM_LAUNCH();
  w.pull = w.deterministic && w.src == w.out;
  if (w.src > w.out) prepare_spans(w, s);
  if (w.pull) det_prepare_pull(w, s);
  if (!w.deterministic && w.src == w.out && w.nunits >= kHotMin) find_hot_rows(w, s);
}

void walk_launch(const TreeWalk &w, const LevelFactors &f, FactorType ft, double *out,
                 cudaStream_t s) {
  if (w.nchunks == 0) return;
  if (w.deterministic && w.src == w.out) {
    launch_pull(w, f, ft, w.src == w.nmodes - 1 ? nullptr : w.src_rows, out, s);
    return;
  }
  const WalkArgs a = make_args(w, &f, w.deterministic && w.out > 0 ? nullptr : out);
  const unsigned blocks = (unsigned)((w.nchunks + kWarps - 1) / kWarps);
  const bool leaf = w.src == w.nmodes - 1;
  if (w.src > w.out) {
    const int vec = vec_for_rank(w.R);
    const int wk = w.walkers > 0 ? w.walkers : default_walkers(w.R);
    if (ft == FactorType::F32) {
      if (leaf) launch_contract<FactorType::F32, true>(vec, wk, w.fold, a, blocks, w.resident, s);
      else launch_contract<FactorType::F32, false>(vec, wk, w.fold, a, blocks, w.resident, s);
    } else {
      if (leaf) launch_contract<FactorType::BF16, true>(vec, wk, w.fold, a, blocks, w.resident, s);
      else launch_contract<FactorType::BF16, false>(vec, wk, w.fold, a, blocks, w.resident, s);
    }
    launch_chains(w, out, s);
    if (w.deterministic && w.out > 0) launch_pull(w, f, ft, w.level_rows.get(), out, s);
  } else {
    const int lanes = lanes_for_rank(w.R);
    if (ft == FactorType::F32) {
      if (leaf) launch_scatter<FactorType::F32, true>(lanes, a, blocks, s);
      else launch_scatter<FactorType::F32, false>(lanes, a, blocks, s);
    } else {
      if (leaf) launch_scatter<FactorType::BF16, true>(lanes, a, blocks, s);
      else launch_scatter<FactorType::BF16, false>(lanes, a, blocks, s);
    }
  }
}

int walk_kernels(const TreeWalk &w) {
  if (w.nchunks == 0) return 0;
  int k = 0;
  if (w.src > w.out) {
    k += 1;                                            // the contraction
    if (w.nchains) k += 1 + (w.nshort ? 1 : 0) + (w.nchains > w.nshort ? 1 : 0);  // chain sums
  }
  if (w.deterministic && w.nsegs) k += w.out + 1 + (w.nlong ? 1 : 0);  // prefix levels, pull, pieces
  if (!w.deterministic && w.src == w.out) k += 1;      // the scatter
  return k;
}

double walk_compulsory_bytes(const TreeWalk &w, FactorType ft, const uint64_t *dims_of_level,
                             uint64_t out_rows) {
  const DevCsf &c = *w.csf;
  const int N = c.nmodes;
  const double R = w.R;
  const double bf = ft == FactorType::F32 ? 4.0 : 2.0;
  double b = 0;
  // structure: every level from 0 to S is traversed
  for (int l = 0; l <= w.src; ++l) {
    b += 4.0 * (double)c.nfibs[l];                         // fids
    if (l < w.src) b += 4.0 * (double)(c.nfibs[l] + 1);    // fptr
  }
  if (w.src == N - 1) b += 4.0 * (double)c.nnz;            // leaf values
  else b += 4.0 * R * (double)c.nfibs[w.src];              // memo rows read
  for (int l = 0; l < N; ++l)
    if (l <= w.src && l != w.out) b += bf * R * (double)dims_of_level[l];  // factors
  for (int l = 0; l < kMaxModes; ++l)
    if (w.store[l]) b += 4.0 * R * (double)c.nfibs[l];     // memo rows written
  b += 8.0 * R * (double)out_rows;                         // output (FP64 rows)
  return b;
}

}  // namespace adatm
