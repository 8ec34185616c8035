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

// Recompute P_l for levels from..d-1.
template <FactorType FT>
__device__ __forceinline__ void prefix_from(const WalkArgs &a, uint32_t *node, float4 *P, int from,
                                            int col, bool act) {
#pragma unroll
  for (int l = 0; l < kMaxModes - 1; ++l) {
    if (l >= from && l < a.d) {
      const float4 row = load_row<FT>(a.U[l], a.fids[l][node[l]], a.ldr, col, act);
      if (l == 0) {
        P[0] = row;
      } else {
        P[l] = f4_mul(P[l > 0 ? l - 1 : 0], row);
      }
    }
  }
}

template <int LANES, FactorType FT, bool LEAF>
__global__ void __launch_bounds__(256) k_contract(const WalkArgs a) {
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t chunk_id = gtid / LANES;
  if (chunk_id >= a.nchunks) return;
  const int t = threadIdx.x % LANES;
  const int col = 4 * t;
  const bool act = col < a.R;
  const unsigned gmask =
      LANES == 32 ? 0xffffffffu : (((1u << LANES) - 1u) << ((threadIdx.x & 31) / LANES * LANES));
  const int S = a.S, d = a.d;

  uint32_t node[kMaxModes], endc[kMaxModes];
  bool part[kMaxModes], touched[kMaxModes];
  float4 acc[kMaxModes], P[kMaxModes];
  const uint32_t *sc = a.sched + (size_t)chunk_id * (S + 1);
  const uint32_t pmask = sc[S];
#pragma unroll
  for (int l = 0; l < kMaxModes; ++l) {
    acc[l] = f4_zero();
    P[l] = f4_zero();
    touched[l] = false;
    part[l] = false;
    node[l] = 0;
    endc[l] = 0;
    if (l < S) {
      node[l] = sc[l];
      endc[l] = a.fptr[l][node[l] + 1];
      part[l] = (pmask >> l) & 1u;
    }
  }
  prefix_from<FT>(a, node, P, 0, col, act);

  const uint64_t u0 = (uint64_t)chunk_id * a.chunk;
  const uint64_t u1 = min(u0 + a.chunk, a.nunits);
  const uint32_t *src_ids = a.src_ids;
  for (uint64_t base = u0; base < u1; base += LANES) {
    const uint64_t mine = base + t;
    uint32_t my_id = 0;
    float my_v = 0.f;
    if (mine < u1) {
      my_id = __ldg(src_ids + mine);
      if constexpr (LEAF) my_v = __ldg(a.vals + mine);
    }
    const int cnt = (int)min((uint64_t)LANES, u1 - base);
    for (int j = 0; j < cnt; ++j) {
      const uint32_t id = __shfl_sync(gmask, my_id, j, LANES);
      const float4 row = load_row<FT>(a.U_src, id, a.ldr, col, act);
      float4 contrib;
      if constexpr (LEAF) {
        const float v = __shfl_sync(gmask, my_v, j, LANES);
        contrib = f4_scale(v, row);
      } else {
        contrib = f4_mul(load_f4(a.src_rows, base + j, a.ldr, col, act), row);
      }
      // add to the level S-1 accumulator
#pragma unroll
      for (int l = 0; l < kMaxModes - 1; ++l)
        if (l == S - 1) {
          f4_add(acc[l], contrib);
          touched[l] = true;
        }
      // completion cascade from level S-1 up
      bool go;
      {
        uint32_t e = 0;
#pragma unroll
        for (int l = 0; l < kMaxModes - 1; ++l)
          if (l == S - 1) e = endc[l];
        go = (uint64_t)(base + j + 1) == (uint64_t)e;
      }
      int pchange = kMaxModes;
#pragma unroll
      for (int l = kMaxModes - 2; l >= 0; --l) {
        if (l < S && go) {
          if (l >= d) {
            const float4 val = acc[l];
            if (a.store[l] != nullptr) {
              if (part[l])
                atomic_f4(a.store[l], node[l], a.ldr, col, val, act);
              else
                store_f4(a.store[l], node[l], a.ldr, col, val, act);
            }
            if (l > d) {
              const float4 r = load_row<FT>(a.U[l], a.fids[l][node[l]], a.ldr, col, act);
              f4_fma(acc[l > 0 ? l - 1 : 0], val, r);
              touched[l > 0 ? l - 1 : 0] = true;
            } else {
              const uint32_t orow = a.fids[l][node[l]];
              if (l == 0) {
                if (part[0])
                  atomic_f4(a.out, orow, a.ldr, col, val, act);
                else
                  store_f4(a.out, orow, a.ldr, col, val, act);
              } else {
                const float4 pv = P[l > 0 ? l - 1 : 0];
                atomic_f4(a.out, orow, a.ldr, col, f4_mul(val, pv), act);
              }
            }
            acc[l] = f4_zero();
            touched[l] = false;
            part[l] = false;
          } else {
            pchange = l;
          }
          node[l] += 1;
          if ((uint64_t)node[l] < a.nfibs[l]) endc[l] = a.fptr[l][node[l] + 1];
          go = (l > 0) && (node[l] == endc[l > 0 ? l - 1 : 0]);
          if (l < d) pchange = l;
        }
      }
      if (pchange < d && (uint64_t)node[0] < a.nfibs[0]) prefix_from<FT>(a, node, P, pchange, col, act);
    }
  }
  // flush the nodes left open by the chunk end
#pragma unroll
  for (int l = kMaxModes - 2; l >= 0; --l) {
    if (l < S && l >= d && touched[l]) {
      const float4 val = acc[l];
      if (a.store[l] != nullptr) atomic_f4(a.store[l], node[l], a.ldr, col, val, act);
      if (l > d) {
        const float4 r = load_row<FT>(a.U[l], a.fids[l][node[l]], a.ldr, col, act);
        f4_fma(acc[l > 0 ? l - 1 : 0], val, r);
        touched[l > 0 ? l - 1 : 0] = true;
      } else {
        const uint32_t orow = a.fids[l][node[l]];
        if (l == 0) {
          atomic_f4(a.out, orow, a.ldr, col, val, act);
        } else {
          const float4 pv = P[l > 0 ? l - 1 : 0];
          atomic_f4(a.out, orow, a.ldr, col, f4_mul(val, pv), act);
        }
      }
    }
  }
}

template <int LANES, FactorType FT, bool LEAF>
__global__ void __launch_bounds__(256) k_scatter(const WalkArgs a) {
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t chunk_id = gtid / LANES;
  if (chunk_id >= a.nchunks) return;
  const int t = threadIdx.x % LANES;
  const int col = 4 * t;
  const bool act = col < a.R;
  const unsigned gmask =
      LANES == 32 ? 0xffffffffu : (((1u << LANES) - 1u) << ((threadIdx.x & 31) / LANES * LANES));
  const int d = a.d;  // == S

  uint32_t node[kMaxModes], endc[kMaxModes];
  float4 P[kMaxModes];
  const uint32_t *sc = a.sched + (size_t)chunk_id * (d + 1);
#pragma unroll
  for (int l = 0; l < kMaxModes; ++l) {
    P[l] = f4_zero();
    node[l] = 0;
    endc[l] = 0;
    if (l < d) {
      node[l] = sc[l];
      endc[l] = a.fptr[l][node[l] + 1];
    }
  }
  prefix_from<FT>(a, node, P, 0, col, act);
  float4 pv = f4_zero();
#pragma unroll
  for (int j2 = 0; j2 < kMaxModes - 1; ++j2)
    if (j2 == d - 1) pv = P[j2];

  const uint64_t u0 = (uint64_t)chunk_id * a.chunk;
  const uint64_t u1 = min(u0 + a.chunk, a.nunits);
  const uint32_t *ids = a.out_ids;
  for (uint64_t base = u0; base < u1; base += LANES) {
    const uint64_t mine = base + t;
    uint32_t my_id = 0;
    float my_v = 0.f;
    if (mine < u1) {
      my_id = __ldg(ids + mine);
      if constexpr (LEAF) my_v = __ldg(a.vals + mine);
    }
    const int cnt = (int)min((uint64_t)LANES, u1 - base);
    for (int j = 0; j < cnt; ++j) {
      const uint32_t id = __shfl_sync(gmask, my_id, j, LANES);
      float4 contrib;
      if constexpr (LEAF) {
        const float v = __shfl_sync(gmask, my_v, j, LANES);
        contrib = f4_scale(v, pv);
      } else {
        contrib = f4_mul(load_f4(a.src_rows, base + j, a.ldr, col, act), pv);
      }
      atomic_f4(a.out, id, a.ldr, col, contrib, act);
      // advance the path above level d
      uint32_t e = 0;
#pragma unroll
      for (int l = 0; l < kMaxModes - 1; ++l)
        if (l == d - 1) e = endc[l];
      bool go = (uint64_t)(base + j + 1) == (uint64_t)e;
      int pchange = kMaxModes;
#pragma unroll
      for (int l = kMaxModes - 2; l >= 0; --l) {
        if (l < d && go) {
          node[l] += 1;
          if ((uint64_t)node[l] < a.nfibs[l]) endc[l] = a.fptr[l][node[l] + 1];
          go = (l > 0) && (node[l] == endc[l > 0 ? l - 1 : 0]);
          pchange = l;
        }
      }
      if (pchange < d && (uint64_t)node[0] < a.nfibs[0] && base + j + 1 < u1) {
        prefix_from<FT>(a, node, P, pchange, col, act);
#pragma unroll
        for (int j2 = 0; j2 < kMaxModes - 1; ++j2)
          if (j2 == d - 1) pv = P[j2];
      }
    }
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
  a.out = out;
  a.sched = w.sched.get();
  return a;
}

template <FactorType FT, bool LEAF, bool CONTRACT>
void launch_lanes(int lanes, const WalkArgs &a, unsigned blocks, cudaStream_t s) {
#define ADATM_WALK_CASE(L)                                                \
  case L:                                                                 \
    if (CONTRACT)                                                         \
      k_contract<L, FT, LEAF><<<blocks, 256, 0, s>>>(a);                  \
    else                                                                  \
      k_scatter<L, FT, LEAF><<<blocks, 256, 0, s>>>(a);                   \
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

void walk_prepare(TreeWalk &w, cudaStream_t s) {
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
