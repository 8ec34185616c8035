// mttkrp.cu -- tree-walk MTTKRP kernels (see mttkrp.cuh for the scheme).
#include <algorithm>

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
  const float *src_rows;
  const uint32_t *src_ids;     // fids of the source level (S)
  const void *U_src;           // factor rows of the source level
  const uint32_t *out_ids;     // fids of the output level (d)
  const uint32_t *par_fptr;    // fptr of level S-1
  const uint32_t *par_fids;    // fids of level S-1
  const void *U_par;           // factor rows of level S-1
  float *par_store;            // memo rows of level S-1 (or null)
  uint64_t par_n;              // nodes of level S-1
  const void *U[kMaxModes];
  float *store[kMaxModes];
  float *out;
  const uint32_t *sched;
};

__device__ __forceinline__ float4 f4_zero() { return make_float4(0.f, 0.f, 0.f, 0.f); }
__device__ __forceinline__ float4 f4_mul(float4 a, float4 b) {
  return make_float4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w);
}
__device__ __forceinline__ float4 f4_scale(float s, float4 a) {
  return make_float4(s * a.x, s * a.y, s * a.z, s * a.w);
}
__device__ __forceinline__ void f4_fma(float4 &acc, float4 a, float4 b) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.y = fmaf(a.y, b.y, acc.y);
  acc.z = fmaf(a.z, b.z, acc.z);
  acc.w = fmaf(a.w, b.w, acc.w);
}
__device__ __forceinline__ void f4_add(float4 &acc, float4 a) {
  acc.x += a.x;
  acc.y += a.y;
  acc.z += a.z;
  acc.w += a.w;
}

template <FactorType FT>
__device__ __forceinline__ float4 load_row(const void *U, uint32_t row, int ldr, int col, bool act) {
  if (!act) return f4_zero();
  if constexpr (FT == FactorType::F32) {
    return __ldg(reinterpret_cast<const float4 *>(static_cast<const float *>(U) + (size_t)row * ldr + col));
  } else {
    const uint2 raw = __ldg(reinterpret_cast<const uint2 *>(
        static_cast<const __nv_bfloat16 *>(U) + (size_t)row * ldr + col));
    const float2 lo = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&raw.x));
    const float2 hi = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&raw.y));
    return make_float4(lo.x, lo.y, hi.x, hi.y);
  }
}

__device__ __forceinline__ float4 load_f4(const float *p, uint64_t row, int ldr, int col, bool act) {
  if (!act) return f4_zero();
  return __ldg(reinterpret_cast<const float4 *>(p + row * (uint64_t)ldr + col));
}

__device__ __forceinline__ void store_f4(float *p, uint64_t row, int ldr, int col, float4 v, bool act) {
  if (act) *reinterpret_cast<float4 *>(p + row * (uint64_t)ldr + col) = v;
}

__device__ __forceinline__ void atomic_f4(float *p, uint64_t row, int ldr, int col, float4 v, bool act) {
  if (act) atomicAdd(reinterpret_cast<float4 *>(p + row * (uint64_t)ldr + col), v);
}

// Units of the source level walked per batch. A batch first stages what it
// needs -- the ids (and values) of its B units, and a window with the ids and
// child ends of the B parent nodes (level S-1) it can touch -- in per-group
// shared memory, then issues all factor-row loads at once (the B unit
// products and the B window rows), and only then walks the units. The walk
// keeps the parent level in registers; the levels above it live in a
// local-memory struct that only the rarer completions of level S-2 touch,
// through out-of-line functions, so the loop body stays small enough for the
// instruction cache. All cross-lane traffic goes through shared memory
// between __syncwarp fences.
constexpr int kBatch = 8;

struct GroupMeta {
  uint32_t id[kBatch];
  float v[kBatch];
  uint32_t wfid[kBatch];
  uint32_t wend[kBatch];
  uint32_t pad;  // 132-byte stride: the groups of a warp start on different banks
};

template <int LANES>
constexpr size_t walk_smem() {
  return (size_t)(256 / LANES) * (2 * kBatch * LANES * sizeof(float4) + sizeof(GroupMeta));
}

// State of the levels above the source's parent level.
struct Upper {
  uint32_t node[kMaxModes];
  uint32_t endc[kMaxModes];
  uint32_t part;     // bit l: the level-l node began before the chunk
  uint32_t touched;  // bit l: acc[l] holds contributions
  float4 acc[kMaxModes];
  float4 P[kMaxModes];  // P_l = U_0[root] * ... * U_l[fids[l][node[l]]]
};

// P_l for levels from..lim-1.
template <FactorType FT>
__device__ __noinline__ void upper_prefix(const WalkArgs &a, Upper &u, int from, int lim, int col,
                                          bool act) {
  for (int l = from; l < lim; ++l) {
    const float4 row = load_row<FT>(a.U[l], a.fids[l][u.node[l]], a.ldr, col, act);
    u.P[l] = l == 0 ? row : f4_mul(u.P[l - 1], row);
  }
}

template <FactorType FT>
__device__ __noinline__ void upper_init(const WalkArgs &a, Upper &u, const uint32_t *sc, int col,
                                        bool act) {
  u.part = sc[a.S];
  u.touched = 0;
  for (int l = 0; l < a.S; ++l) {
    u.node[l] = sc[l];
    u.endc[l] = a.fptr[l][u.node[l] + 1];
    u.acc[l] = f4_zero();
  }
  upper_prefix<FT>(a, u, 0, min(a.d, a.S - 1), col, act);
}

// The node of level p = S-2 completed; its sum is accP (or u.acc). Emit it and
// every ancestor that completes with it; advance the path; refresh P.
template <FactorType FT>
__device__ __noinline__ void upper_complete(const WalkArgs &a, Upper &u, float4 accP, int col,
                                            bool act) {
  const int d = a.d;
  int pchange = kMaxModes;
  bool carry = true;
  for (int l = a.S - 2; l >= 0 && carry; --l) {
    if (l >= d) {
      const float4 v = (l == a.S - 2) ? accP : u.acc[l];
      const bool part = (u.part >> l) & 1u;
      if (a.store[l] != nullptr) {
        if (part) atomic_f4(a.store[l], u.node[l], a.ldr, col, v, act);
        else store_f4(a.store[l], u.node[l], a.ldr, col, v, act);
      }
      if (l > d) {
        const float4 r = load_row<FT>(a.U[l], a.fids[l][u.node[l]], a.ldr, col, act);
        f4_fma(u.acc[l - 1], v, r);
        u.touched |= 1u << (l - 1);
      } else {
        const uint32_t orow = a.fids[l][u.node[l]];
        if (l == 0) {
          if (part) atomic_f4(a.out, orow, a.ldr, col, v, act);
          else store_f4(a.out, orow, a.ldr, col, v, act);
        } else {
          atomic_f4(a.out, orow, a.ldr, col, f4_mul(v, u.P[l - 1]), act);
        }
      }
      u.acc[l] = f4_zero();
      u.touched &= ~(1u << l);
      u.part &= ~(1u << l);
    } else {
      pchange = l;
    }
    u.node[l] += 1;
    if ((uint64_t)u.node[l] < a.nfibs[l]) u.endc[l] = a.fptr[l][u.node[l] + 1];
    carry = l > 0 && u.node[l] == u.endc[l - 1];
  }
  if (pchange < kMaxModes && (uint64_t)u.node[0] < a.nfibs[0])
    upper_prefix<FT>(a, u, pchange, min(d, a.S - 1), col, act);
}

// Chunk end: the open nodes of levels d..S-2 get their partial sums added.
template <FactorType FT>
__device__ __noinline__ void upper_flush(const WalkArgs &a, Upper &u, float4 accP, bool touchP,
                                         int col, bool act) {
  const int d = a.d;
  const int p = a.S - 2;
  if (p >= d && touchP) {
    u.acc[p] = accP;
    u.touched |= 1u << p;
  }
  for (int l = p; l >= d; --l) {
    if (!((u.touched >> l) & 1u)) continue;
    const float4 v = u.acc[l];
    if (a.store[l] != nullptr) atomic_f4(a.store[l], u.node[l], a.ldr, col, v, act);
    if (l > d) {
      const float4 r = load_row<FT>(a.U[l], a.fids[l][u.node[l]], a.ldr, col, act);
      f4_fma(u.acc[l - 1], v, r);
      u.touched |= 1u << (l - 1);
    } else {
      const uint32_t orow = a.fids[l][u.node[l]];
      atomic_f4(a.out, orow, a.ldr, col, l == 0 ? v : f4_mul(v, u.P[l - 1]), act);
    }
  }
}

// Stage one batch: unit ids/values and the parent window into meta, then
// the unit products (or memo rows) into cbuf and the window's factor rows
// into fbuf. Returns with the group fenced.
template <int LANES, FactorType FT, bool LEAF, bool CONTRIB>
__device__ __forceinline__ void issue_batch(const WalkArgs &a, uint64_t base, int cnt, int t,
                                            int col, bool act, unsigned gmask, uint32_t nodeS,
                                            uint64_t FS, bool want_rows, float4 *cbuf,
                                            float4 *fbuf, GroupMeta *meta) {
  constexpr int B = kBatch;
  for (int k = t; k < B; k += LANES) {
    uint32_t id = 0;
    float v = 0.f;
    if (k < cnt) {
      id = __ldg(a.src_ids + base + k);
      if constexpr (LEAF) v = __ldg(a.vals + base + k);
    }
    meta->id[k] = id;
    meta->v[k] = v;
    const uint64_t n = (uint64_t)nodeS + k;
    const bool in = n < FS;
    meta->wfid[k] = in ? __ldg(a.par_fids + n) : 0u;
    meta->wend[k] = in ? __ldg(a.par_fptr + n + 1) : 0u;
  }
  __syncwarp(gmask);
#pragma unroll
  for (int k = 0; k < B; ++k) {
    if (k < cnt) {
      if constexpr (CONTRIB) {
        const float4 row = load_row<FT>(a.U_src, meta->id[k], a.ldr, col, act);
        if constexpr (LEAF) {
          cbuf[k * LANES + t] = f4_scale(meta->v[k], row);
        } else {
          cbuf[k * LANES + t] = f4_mul(load_f4(a.src_rows, base + k, a.ldr, col, act), row);
        }
      } else if constexpr (!LEAF) {
        cbuf[k * LANES + t] = load_f4(a.src_rows, base + k, a.ldr, col, act);
      }
    }
  }
  if (want_rows) {
#pragma unroll
    for (int k = 0; k < B; ++k)
      if ((uint64_t)nodeS + k < FS)
        fbuf[k * LANES + t] = load_row<FT>(a.U_par, meta->wfid[k], a.ldr, col, act);
  }
}

template <int LANES, FactorType FT, bool LEAF>
__global__ void __launch_bounds__(256) k_contract(const __grid_constant__ WalkArgs a) {
  constexpr int B = kBatch;
  extern __shared__ float4 wsm[];
  const uint32_t chunk_id = (blockIdx.x * blockDim.x + threadIdx.x) / LANES;
  if (chunk_id >= a.nchunks) return;
  const int t = threadIdx.x % LANES;
  const int grp = threadIdx.x / LANES;
  float4 *cbuf = wsm + (size_t)grp * 2 * B * LANES;
  float4 *fbuf = cbuf + B * LANES;
  GroupMeta *meta = reinterpret_cast<GroupMeta *>(wsm + (size_t)(256 / LANES) * 2 * B * LANES) + grp;
  const int col = 4 * t;
  const bool act = col < a.R;
  const unsigned gmask =
      LANES == 32 ? 0xffffffffu : (((1u << LANES) - 1u) << ((threadIdx.x & 31) / LANES * LANES));
  const int d = a.d, L1 = a.S - 1;
  const uint32_t *sc = a.sched + (size_t)chunk_id * (a.S + 1);
  Upper u;
  upper_init<FT>(a, u, sc, col, act);
  const uint64_t FS = a.par_n;
  uint32_t nodeS = sc[L1];
  uint32_t endS = a.par_fptr[nodeS + 1];
  bool partS = (sc[a.S] >> L1) & 1u;
  uint32_t endP = L1 > 0 ? u.endc[L1 - 1] : 0xffffffffu;
  float4 pv = (L1 == d && d > 0) ? u.P[d - 1] : f4_zero();
  float4 accS = f4_zero(), accP = f4_zero();
  bool touchS = false, touchP = false;
  int w = 0;
  uint32_t open_fid = 0;  // id of the open parent node at the chunk end
  const uint64_t u0 = (uint64_t)chunk_id * a.chunk;
  const uint64_t u1 = min(u0 + a.chunk, a.nunits);
  for (uint64_t base = u0; base < u1; base += B) {
    const int cnt = (int)min((uint64_t)B, u1 - base);
    issue_batch<LANES, FT, LEAF, true>(a, base, cnt, t, col, act, gmask, nodeS, FS, L1 > d, cbuf,
                                       fbuf, meta);
    w = 0;
    for (int k = 0; k < cnt; ++k) {
      f4_add(accS, cbuf[k * LANES + t]);
      touchS = true;
      if (base + k + 1 != (uint64_t)endS) continue;
      // the parent (level S-1) node is complete
      const float4 val = accS;
      accS = f4_zero();
      touchS = false;
      const bool was_part = partS;
      partS = false;
      if (a.par_store != nullptr) {
        if (was_part) atomic_f4(a.par_store, nodeS, a.ldr, col, val, act);
        else store_f4(a.par_store, nodeS, a.ldr, col, val, act);
      }
      if (L1 > d) {
        f4_fma(accP, val, fbuf[w * LANES + t]);
        touchP = true;
      } else {
        const uint32_t orow = meta->wfid[w];
        if (d == 0) {
          if (was_part) atomic_f4(a.out, orow, a.ldr, col, val, act);
          else store_f4(a.out, orow, a.ldr, col, val, act);
        } else {
          atomic_f4(a.out, orow, a.ldr, col, f4_mul(val, pv), act);
        }
      }
      ++w;
      ++nodeS;
      if (w < B) endS = meta->wend[w];
      else if ((uint64_t)nodeS < FS) endS = __ldg(a.par_fptr + nodeS + 1);
      if (L1 > 0 && nodeS == endP) {
        upper_complete<FT>(a, u, accP, col, act);
        accP = f4_zero();
        touchP = false;
        endP = u.endc[L1 - 1];
        if (L1 == d && d > 0) pv = u.P[d - 1];
      }
    }
    if (touchS) open_fid = meta->wfid[w < B ? w : B - 1];
    __syncwarp(gmask);
  }
  if (touchS) {
    if (a.par_store != nullptr) atomic_f4(a.par_store, nodeS, a.ldr, col, accS, act);
    if (L1 > d) {
      // the open parent node is window entry w of the last batch (w < B: it has units)
      f4_fma(accP, accS, fbuf[w * LANES + t]);
      touchP = true;
    } else {
      atomic_f4(a.out, open_fid, a.ldr, col, d == 0 ? accS : f4_mul(accS, pv), act);
    }
  }
  if (L1 - 1 >= d) upper_flush<FT>(a, u, accP, touchP, col, act);
}

template <int LANES, FactorType FT, bool LEAF>
__global__ void __launch_bounds__(256) k_scatter(const __grid_constant__ WalkArgs a) {
  constexpr int B = kBatch;
  extern __shared__ float4 wsm[];
  const uint32_t chunk_id = (blockIdx.x * blockDim.x + threadIdx.x) / LANES;
  if (chunk_id >= a.nchunks) return;
  const int t = threadIdx.x % LANES;
  const int grp = threadIdx.x / LANES;
  float4 *cbuf = wsm + (size_t)grp * 2 * B * LANES;
  float4 *fbuf = cbuf + B * LANES;
  GroupMeta *meta = reinterpret_cast<GroupMeta *>(wsm + (size_t)(256 / LANES) * 2 * B * LANES) + grp;
  const int col = 4 * t;
  const bool act = col < a.R;
  const unsigned gmask =
      LANES == 32 ? 0xffffffffu : (((1u << LANES) - 1u) << ((threadIdx.x & 31) / LANES * LANES));
  const int L1 = a.S - 1;  // parent level of the units; the output level is S
  const uint32_t *sc = a.sched + (size_t)chunk_id * (a.S + 1);
  Upper u;
  upper_init<FT>(a, u, sc, col, act);
  const uint64_t FS = a.par_n;
  uint32_t nodeS = sc[L1];
  uint32_t endS = a.par_fptr[nodeS + 1];
  uint32_t endP = L1 > 0 ? u.endc[L1 - 1] : 0xffffffffu;
  float4 above = L1 > 0 ? u.P[L1 - 1] : make_float4(1.f, 1.f, 1.f, 1.f);
  const uint64_t u0 = (uint64_t)chunk_id * a.chunk;
  const uint64_t u1 = min(u0 + a.chunk, a.nunits);
  for (uint64_t base = u0; base < u1; base += B) {
    const int cnt = (int)min((uint64_t)B, u1 - base);
    issue_batch<LANES, FT, LEAF, false>(a, base, cnt, t, col, act, gmask, nodeS, FS, true, cbuf,
                                        fbuf, meta);
    int w = 0;
    float4 pv = f4_mul(above, fbuf[t]);
    for (int k = 0; k < cnt; ++k) {
      float4 c;
      if constexpr (LEAF) c = f4_scale(meta->v[k], pv);
      else c = f4_mul(cbuf[k * LANES + t], pv);
      atomic_f4(a.out, meta->id[k], a.ldr, col, c, act);
      if (base + k + 1 != (uint64_t)endS) continue;
      ++w;
      ++nodeS;
      if (w < B) endS = meta->wend[w];
      else if ((uint64_t)nodeS < FS) endS = __ldg(a.par_fptr + nodeS + 1);
      if (L1 > 0 && nodeS == endP) {
        upper_complete<FT>(a, u, f4_zero(), col, act);
        endP = u.endc[L1 - 1];
        above = u.P[L1 - 1];
      }
      if (w < B) pv = f4_mul(above, fbuf[w * LANES + t]);
    }
    __syncwarp(gmask);
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

// Zero the memo rows that chunk boundaries cut (they are filled by atomics).
__global__ void k_prezero(WalkArgs a, const uint32_t *sched) {
  const uint32_t c = blockIdx.x * blockDim.y + threadIdx.y;
  if (c >= a.nchunks || c == 0) return;
  const int S = a.S;
  const uint32_t mask = sched[(size_t)c * (S + 1) + S];
  for (int l = a.d; l < S; ++l) {
    if (a.store[l] == nullptr || !((mask >> l) & 1u)) continue;
    const uint32_t n = sched[(size_t)c * (S + 1) + l];
    for (int r = threadIdx.x; r < a.ldr; r += blockDim.x) a.store[l][(size_t)n * a.ldr + r] = 0.f;
  }
}

WalkArgs make_args(const TreeWalk &w, const LevelFactors *f, float *out) {
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
  a.out_ids = c.fids[w.out].get();
  a.U_src = f ? f->U[w.src] : nullptr;
  const int par = w.src > 0 ? w.src - 1 : 0;
  a.par_fptr = c.fptr[par].get();
  a.par_fids = c.fids[par].get();
  a.U_par = f ? f->U[par] : nullptr;
  a.par_store = w.store[par];
  a.par_n = c.nfibs[par];
  a.out = out;
  a.sched = w.sched.get();
  return a;
}

template <FactorType FT, bool LEAF, bool CONTRACT>
void launch_lanes(int lanes, const WalkArgs &a, unsigned blocks, cudaStream_t s) {
#define ADATM_WALK_CASE(L)                                                \
  case L:                                                                 \
    if (CONTRACT)                                                         \
      k_contract<L, FT, LEAF><<<blocks, 256, walk_smem<L>(), s>>>(a); \
    else                                                                  \
      k_scatter<L, FT, LEAF><<<blocks, 256, walk_smem<L>(), s>>>(a);     \
    break;
  switch (lanes) {
    ADATM_WALK_CASE(4)
    ADATM_WALK_CASE(8)
    ADATM_WALK_CASE(16)
    ADATM_WALK_CASE(32)
    default: throw BadInput("unsupported lane count");
  }
#undef ADATM_WALK_CASE
  ADATM_LAUNCH();
}

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
#define ADATM_ATTR(L, FT, LEAF)                                                           \
  ADATM_CUDA(cudaFuncSetAttribute(k_contract<L, FT, LEAF>,                                \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,            \
                                  (int)walk_smem<L>()));                                  \
  ADATM_CUDA(cudaFuncSetAttribute(k_scatter<L, FT, LEAF>,                                 \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,            \
                                  (int)walk_smem<L>()));
#define ADATM_ATTR_L(L)                        \
  ADATM_ATTR(L, FactorType::F32, true)         \
  ADATM_ATTR(L, FactorType::F32, false)        \
  ADATM_ATTR(L, FactorType::BF16, true)        \
  ADATM_ATTR(L, FactorType::BF16, false)
  ADATM_ATTR_L(4)
  ADATM_ATTR_L(8)
  ADATM_ATTR_L(16)
  ADATM_ATTR_L(32)
#undef ADATM_ATTR_L
#undef ADATM_ATTR
  done = true;
}

void walk_prepare(TreeWalk &w, cudaStream_t s) {
  set_walk_attributes();
  const DevCsf &c = *w.csf;
  w.nmodes = c.nmodes;
  w.nunits = c.nfibs[w.src];
  if (w.chunk == 0) w.chunk = 32;
  w.nchunks = (uint32_t)((w.nunits + w.chunk - 1) / w.chunk);
  w.sched.alloc((size_t)std::max<uint32_t>(w.nchunks, 1) * (w.src + 1));
  if (w.nchunks == 0) return;
  WalkArgs a = make_args(w, nullptr, nullptr);
  k_schedule<<<(w.nchunks + 255) / 256, 256, 0, s>>>(a, w.sched.get());
  ADATM_LAUNCH();
}

void walk_launch(const TreeWalk &w, const LevelFactors &f, FactorType ft, float *out,
                 cudaStream_t s) {
  if (w.nchunks == 0) return;
  const WalkArgs a = make_args(w, &f, out);
  if (w.has_store()) {
    dim3 blk(32, 8);
    k_prezero<<<(w.nchunks + 7) / 8, blk, 0, s>>>(a, w.sched.get());
    ADATM_LAUNCH();
  }
  const int lanes = lanes_for_rank(w.R);
  const unsigned blocks = (unsigned)(((uint64_t)w.nchunks * lanes + 255) / 256);
  const bool leaf = w.src == w.nmodes - 1;
  const bool contract = w.src > w.out;
  if (ft == FactorType::F32) {
    if (leaf && contract) launch_lanes<FactorType::F32, true, true>(lanes, a, blocks, s);
    else if (leaf) launch_lanes<FactorType::F32, true, false>(lanes, a, blocks, s);
    else if (contract) launch_lanes<FactorType::F32, false, true>(lanes, a, blocks, s);
    else launch_lanes<FactorType::F32, false, false>(lanes, a, blocks, s);
  } else {
    if (leaf && contract) launch_lanes<FactorType::BF16, true, true>(lanes, a, blocks, s);
    else if (leaf) launch_lanes<FactorType::BF16, true, false>(lanes, a, blocks, s);
    else if (contract) launch_lanes<FactorType::BF16, false, true>(lanes, a, blocks, s);
    else launch_lanes<FactorType::BF16, false, false>(lanes, a, blocks, s);
  }
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
  b += 4.0 * R * (double)out_rows;                         // output
  return b;
}

}  // namespace adatm
