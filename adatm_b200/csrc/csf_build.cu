// csf_build.cu -- GPU construction of CSF trees (the reference builds them
// serially on the host in p_csf_alloc_untiled, adatm_rcsf.c:173-209).
//
// Pipeline for one tree with level order `perm`:
//  1. pack every nonzero's coordinates into a 64..192-bit key, root level in
//     the most significant bits (k_pack);
//  2. stable LSD radix sort of (key, position) with 8-bit digits; each pass is
//     a tile histogram, a device scan of the digit-major counts, and a
//     scatter that ranks each tile stably with warp match_any and writes the
//     tile bucket by bucket through shared memory;
//  3. per tile, count the new-node flags of every level (a node opens at
//     level l where any of the coordinates of levels 0..l changes), scan
//     them per level;
//  4. fill fptr/fids/vals in one pass: a level-l node opening at position n
//     gets the next level-l id; its fptr entry is the id of the level-(l+1)
//     node opening at n (or n itself for l = N-2).
// No kernel waits on another block; every phase is a separate launch.
#include <cmath>
#include <vector>

#include "csf_build.cuh"

namespace adatm {

size_t DevCsf::device_bytes() const {
  size_t b = vals64.bytes() + vals32.bytes();
  for (int l = 0; l < kMaxModes; ++l) b += fptr[l].bytes() + fids[l].bytes() + cdepth[l].bytes();
  return b;
}

static int bitwidth(uint64_t v) {
  int b = 0;
  while (v) {
    ++b;
    v >>= 1;
  }
  return b;
}

KeySpec make_key_spec(int nmodes, const uint64_t *dims, const uint64_t *perm) {
  KeySpec k;
  k.nlev = nmodes;
  int word = 0, used = 0;
  for (int l = nmodes - 1; l >= 0; --l) {
    const int b = bitwidth(dims[perm[l]] > 0 ? dims[perm[l]] - 1 : 0);
    if (used + b > 64) {
      ++word;
      used = 0;
      if (word >= 3) throw BadInput("coordinate key wider than 192 bits");
    }
    k.word[l] = word;
    k.shift[l] = used;
    k.bits[l] = b;
    used += b;
    k.used_bits[word] = used;
  }
  k.words = word + 1;
  for (int l = 0; l < nmodes; ++l)
    for (int j = 0; j <= l; ++j)
      if (k.bits[j] > 0) k.prefix_mask[l][k.word[j]] |= ((1ull << k.bits[j]) - 1ull) << k.shift[j];
  return k;
}

namespace {

template <int W>
struct Key {
  uint64_t w[W];
};

struct IdxPtrs {
  const uint32_t *p[kMaxModes];
};

template <int W>
__device__ __forceinline__ uint32_t key_field(const Key<W> &k, const KeySpec &s, int l) {
  uint64_t v = 0;
#pragma unroll
  for (int w = 0; w < W; ++w)
    if (s.word[l] == w) v = k.w[w];
  const int b = s.bits[l];
  return b == 0 ? 0u : (uint32_t)((v >> s.shift[l]) & ((1ull << b) - 1ull));
}

template <int W>
__device__ __forceinline__ bool prefix_differs(const Key<W> &a, const Key<W> &b, const KeySpec &s,
                                               int l) {
  uint64_t d = 0;
#pragma unroll
  for (int w = 0; w < W; ++w) d |= (a.w[w] ^ b.w[w]) & s.prefix_mask[l][w];
  return d != 0;
}

template <int W>
__device__ __forceinline__ bool key_equal(const Key<W> &a, const Key<W> &b) {
  bool e = true;
#pragma unroll
  for (int w = 0; w < W; ++w) e = e && (a.w[w] == b.w[w]);
  return e;
}

// ---------------------------------------------------------------------------
// 1. key packing
// ---------------------------------------------------------------------------
template <int W>
__global__ void k_pack(IdxPtrs idx, KeySpec spec, uint64_t n, Key<W> *keys, uint32_t *order) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Key<W> k;
#pragma unroll
  for (int w = 0; w < W; ++w) k.w[w] = 0;
  for (int l = 0; l < spec.nlev; ++l) {
    const uint64_t v = idx.p[l][i];
#pragma unroll
    for (int w = 0; w < W; ++w)
      if (spec.word[l] == w) k.w[w] |= v << spec.shift[l];
  }
  keys[i] = k;
  order[i] = (uint32_t)i;
}

// ---------------------------------------------------------------------------
// 2. radix sort
// ---------------------------------------------------------------------------
constexpr int kRsThreads = 256;
constexpr int kRsWarps = kRsThreads / 32;

template <int W>
struct RsTile {
  static constexpr int items = W == 1 ? 16 : (W == 2 ? 12 : 8);  // per lane
  static constexpr int tile = kRsThreads * items;
  static constexpr size_t smem = (size_t)tile * (sizeof(Key<W>) + sizeof(uint32_t));
};

template <int W>
__device__ __forceinline__ int rs_digit(const Key<W> &k, int word, int shift) {
  uint64_t v = 0;
#pragma unroll
  for (int w = 0; w < W; ++w)
    if (word == w) v = k.w[w];
  return (int)((v >> shift) & 0xFFu);
}

template <int W>
__global__ void __launch_bounds__(kRsThreads) k_rs_hist(const Key<W> *keys, uint64_t n, int word,
                                                        int shift, uint32_t *counts,
                                                        uint32_t ntiles) {
  __shared__ uint32_t hist[256];
  hist[threadIdx.x] = 0;
  __syncthreads();
  const uint64_t base = (uint64_t)blockIdx.x * RsTile<W>::tile;
  const uint64_t end = min(base + (uint64_t)RsTile<W>::tile, n);
  for (uint64_t i = base + threadIdx.x; i < end; i += kRsThreads)
    atomicAdd(&hist[rs_digit<W>(keys[i], word, shift)], 1u);
  __syncthreads();
  counts[(size_t)threadIdx.x * ntiles + blockIdx.x] = hist[threadIdx.x];
}

template <int W>
__global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const Key<W> *__restrict__ kin,
                                                           const uint32_t *__restrict__ oin,
                                                           Key<W> *__restrict__ kout,
                                                           uint32_t *__restrict__ oout, uint64_t n,
                                                           int word, int shift,
                                                           const uint32_t *__restrict__ offsets,
                                                           uint32_t ntiles) {
  constexpr int IT = RsTile<W>::items;
  constexpr int TILE = RsTile<W>::tile;
  extern __shared__ __align__(16) unsigned char rs_smem[];
  Key<W> *skey = reinterpret_cast<Key<W> *>(rs_smem);
  uint32_t *sord = reinterpret_cast<uint32_t *>(rs_smem + (size_t)TILE * sizeof(Key<W>));
  __shared__ uint32_t whist[kRsWarps][256];
  __shared__ uint32_t tile_off[256];
  __shared__ uint32_t glob_off[256];
  __shared__ uint32_t scan_tmp[kRsWarps];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < kRsWarps * 256; i += kRsThreads) (&whist[0][0])[i] = 0;
  __syncthreads();

  const uint64_t base = (uint64_t)blockIdx.x * TILE;
  const uint64_t wbase = base + (uint64_t)warp * 32 * IT;
  Key<W> k[IT];
  uint32_t o[IT];
  uint32_t rank[IT];
  int dig[IT];
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int r = 0; r < IT; ++r) {
    const uint64_t i = wbase + (uint64_t)r * 32 + lane;
    const bool valid = i < n;
    if (valid) {
      k[r] = kin[i];
      o[r] = oin[i];
      dig[r] = rs_digit<W>(k[r], word, shift);
    } else {
      dig[r] = 256;
    }
    const uint32_t peers = __match_any_sync(0xffffffffu, dig[r]);
    const uint32_t pre = valid ? whist[warp][dig[r]] : 0u;
    __syncwarp();
    rank[r] = pre + __popc(peers & lt);
    if (valid && lane == __ffs(peers) - 1) whist[warp][dig[r]] = pre + __popc(peers);
    __syncwarp();
  }
  __syncthreads();

  // per digit: offsets of each warp inside the tile's bucket, tile totals
  {
    const int d = tid;
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kRsWarps; ++w) {
      const uint32_t t = whist[w][d];
      whist[w][d] = run;
      run += t;
    }
    // block exclusive scan of run over the 256 digits
    uint32_t v = run;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, v, off);
      if (lane >= off) v += t;
    }
    if (lane == 31) scan_tmp[warp] = v;
    __syncthreads();
    if (warp == 0) {
      uint32_t s = lane < kRsWarps ? scan_tmp[lane] : 0u;
      uint32_t si = s;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, si, off);
        if (lane >= off) si += t;
      }
      if (lane < kRsWarps) scan_tmp[lane] = si - s;
    }
    __syncthreads();
    tile_off[d] = scan_tmp[warp] + v - run;
    glob_off[d] = offsets[(size_t)d * ntiles + blockIdx.x];
  }
  __syncthreads();

#pragma unroll
  for (int r = 0; r < IT; ++r) {
    if (dig[r] < 256) {
      const uint32_t pos = tile_off[dig[r]] + whist[warp][dig[r]] + rank[r];
      skey[pos] = k[r];
      sord[pos] = o[r];
    }
  }
  __syncthreads();

  const uint32_t tile_n = (uint32_t)min((uint64_t)TILE, n - base);
  for (uint32_t i = tid; i < tile_n; i += kRsThreads) {
    const Key<W> kk = skey[i];
    const int d = rs_digit<W>(kk, word, shift);
    const uint32_t dst = glob_off[d] + (i - tile_off[d]);
    kout[dst] = kk;
    oout[dst] = sord[i];
  }
}

template <int W>
struct SortBufs {
  DevBuf<Key<W>> k0, k1;
  DevBuf<uint32_t> o0, o1;
  Key<W> *keys = nullptr;   // sorted result
  uint32_t *order = nullptr;
};

// Sort keys (packed from `coo` under `spec`) stably; result in b.keys/b.order.
template <int W>
void sort_keys(const DevCoo &coo, const uint64_t *perm, const KeySpec &spec, SortBufs<W> &b,
               cudaStream_t s) {
  const uint64_t n = coo.nnz;
  b.k0.alloc(n);
  b.k1.alloc(n);
  b.o0.alloc(n);
  b.o1.alloc(n);
  IdxPtrs ip;
  for (int l = 0; l < kMaxModes; ++l) ip.p[l] = nullptr;
  for (int l = 0; l < coo.nmodes; ++l) ip.p[l] = coo.idx[perm[l]].get();
  const unsigned blocks = (unsigned)((n + 255) / 256);
  k_pack<W><<<blocks, 256, 0, s>>>(ip, spec, n, b.k0.get(), b.o0.get());
  ADATM_LAUNCH();
  const uint32_t ntiles = (uint32_t)((n + RsTile<W>::tile - 1) / RsTile<W>::tile);
  DevBuf<uint32_t> counts((size_t)256 * ntiles), offs((size_t)256 * ntiles),
      tmp(scan_tmp_words((size_t)256 * ntiles));
  ADATM_CUDA(cudaFuncSetAttribute(k_rs_scatter<W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)RsTile<W>::smem));
  Key<W> *kin = b.k0.get(), *kout = b.k1.get();
  uint32_t *oin = b.o0.get(), *oout = b.o1.get();
  for (int w = 0; w < spec.words; ++w) {
    for (int sh = 0; sh < spec.used_bits[w]; sh += 8) {
      k_rs_hist<W><<<ntiles, kRsThreads, 0, s>>>(kin, n, w, sh, counts.get(), ntiles);
      ADATM_LAUNCH();
      exclusive_scan_u32(counts.get(), offs.get(), (size_t)256 * ntiles, tmp.get(), s);
      k_rs_scatter<W><<<ntiles, kRsThreads, RsTile<W>::smem, s>>>(kin, oin, kout, oout, n, w, sh,
                                                                  offs.get(), ntiles);
      ADATM_LAUNCH();
      std::swap(kin, kout);
      std::swap(oin, oout);
    }
  }
  b.keys = kin;
  b.order = oin;
}

// ---------------------------------------------------------------------------
// 3./4. level flags, counts and fill
// ---------------------------------------------------------------------------
constexpr int kLvThreads = 256;
constexpr int kLvItems = 16;
constexpr int kLvTile = kLvThreads * kLvItems;

// Per tile, count how many nodes open at every level 0..N-2.
template <int W>
__global__ void __launch_bounds__(kLvThreads) k_level_count(const Key<W> *keys, uint64_t n,
                                                            KeySpec spec, uint32_t *counts,
                                                            uint32_t ntiles) {
  const int nl = spec.nlev - 1;
  uint32_t cnt[kMaxModes];
#pragma unroll
  for (int l = 0; l < kMaxModes; ++l) cnt[l] = 0;
  const uint64_t start = (uint64_t)blockIdx.x * kLvTile + (uint64_t)threadIdx.x * kLvItems;
  Key<W> prev;
  if (start > 0 && start < n) prev = keys[start - 1];
  for (int e = 0; e < kLvItems; ++e) {
    const uint64_t i = start + e;
    if (i >= n) break;
    const Key<W> cur = keys[i];
#pragma unroll
    for (int l = 0; l < kMaxModes - 1; ++l)
      if (l < nl && (i == 0 || prefix_differs<W>(cur, prev, spec, l))) ++cnt[l];
    prev = cur;
  }
  __shared__ uint32_t red[kLvThreads / 32][kMaxModes];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int l = 0; l < kMaxModes - 1; ++l) {
    uint32_t v = cnt[l];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) red[warp][l] = v;
  }
  __syncthreads();
  if (threadIdx.x < (unsigned)nl) {
    uint32_t t = 0;
    for (int w = 0; w < kLvThreads / 32; ++w) t += red[w][threadIdx.x];
    counts[(size_t)threadIdx.x * ntiles + blockIdx.x] = t;
  }
}

__global__ void k_level_totals(const uint32_t *counts, const uint32_t *offs, uint32_t ntiles,
                               int nl, uint32_t *totals) {
  const int l = threadIdx.x;
  if (l < nl) {
    const size_t last = (size_t)l * ntiles + ntiles - 1;
    totals[l] = offs[last] + counts[last];
  }
}

struct LevelOut {
  uint32_t *fptr[kMaxModes];
  uint32_t *fids[kMaxModes];
};

template <int W>
__global__ void __launch_bounds__(kLvThreads) k_level_fill(const Key<W> *keys,
                                                           const uint32_t *order, uint64_t n,
                                                           KeySpec spec, const uint32_t *offs,
                                                           uint32_t ntiles, LevelOut out,
                                                           const double *vals_in, double *vals64,
                                                           float *vals32) {
  const int N = spec.nlev;
  const int nl = N - 1;
  uint32_t cnt[kMaxModes];
#pragma unroll
  for (int l = 0; l < kMaxModes; ++l) cnt[l] = 0;
  const uint64_t start = (uint64_t)blockIdx.x * kLvTile + (uint64_t)threadIdx.x * kLvItems;
  Key<W> prev;
  if (start > 0 && start < n) prev = keys[start - 1];
  {
    Key<W> p2 = prev;
    for (int e = 0; e < kLvItems; ++e) {
      const uint64_t i = start + e;
      if (i >= n) break;
      const Key<W> cur = keys[i];
#pragma unroll
      for (int l = 0; l < kMaxModes - 1; ++l)
        if (l < nl && (i == 0 || prefix_differs<W>(cur, p2, spec, l))) ++cnt[l];
      p2 = cur;
    }
  }
  // block exclusive scan of every level's count
  __shared__ uint32_t wsum[kLvThreads / 32][kMaxModes];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t run[kMaxModes];
#pragma unroll
  for (int l = 0; l < kMaxModes - 1; ++l) {
    uint32_t v = cnt[l];
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, v, off);
      if (lane >= off) v += t;
    }
    run[l] = v - cnt[l];
    if (lane == 31) wsum[warp][l] = v;
  }
  __syncthreads();
#pragma unroll
  for (int l = 0; l < kMaxModes - 1; ++l) {
    if (l < nl) {
      uint32_t add = offs[(size_t)l * ntiles + blockIdx.x];
      for (int w = 0; w < warp; ++w) add += wsum[w][l];
      run[l] += add;
    }
  }
  for (int e = 0; e < kLvItems; ++e) {
    const uint64_t i = start + e;
    if (i >= n) break;
    const Key<W> cur = keys[i];
    bool flag[kMaxModes];
#pragma unroll
    for (int l = 0; l < kMaxModes - 1; ++l)
      flag[l] = l < nl && (i == 0 || prefix_differs<W>(cur, prev, spec, l));
#pragma unroll
    for (int l = 0; l < kMaxModes - 1; ++l) {
      if (flag[l]) {
        const uint32_t node = run[l];
        out.fids[l][node] = key_field<W>(cur, spec, l);
        uint32_t child = (uint32_t)i;
#pragma unroll
        for (int j = 1; j < kMaxModes - 1; ++j)
          if (j == l + 1 && l + 1 < nl) child = run[j];
        out.fptr[l][node] = child;
      }
    }
#pragma unroll
    for (int l = 0; l < kMaxModes - 1; ++l)
      if (flag[l]) ++run[l];
    out.fids[N - 1][i] = key_field<W>(cur, spec, N - 1);
    const double v = vals_in[order[i]];
    vals64[i] = v;
    vals32[i] = (float)v;
    prev = cur;
  }
}

__global__ void k_level_tails(LevelOut out, const uint32_t *totals, int nl, uint64_t n) {
  const int l = threadIdx.x;
  if (l < nl) out.fptr[l][totals[l]] = (l + 1 < nl) ? totals[l + 1] : (uint32_t)n;
}

template <int W>
void count_levels(const SortBufs<W> &b, uint64_t n, const KeySpec &spec, DevBuf<uint32_t> &offs,
                  uint32_t &ntiles, uint64_t *nfibs, cudaStream_t s) {
  const int nl = spec.nlev - 1;
  ntiles = (uint32_t)((n + kLvTile - 1) / kLvTile);
  DevBuf<uint32_t> counts((size_t)nl * ntiles), tmp(scan_tmp_words(ntiles)), totals(kMaxModes);
  offs.alloc((size_t)nl * ntiles);
  k_level_count<W><<<ntiles, kLvThreads, 0, s>>>(b.keys, n, spec, counts.get(), ntiles);
  ADATM_LAUNCH();
  for (int l = 0; l < nl; ++l)
    exclusive_scan_u32(counts.get() + (size_t)l * ntiles, offs.get() + (size_t)l * ntiles, ntiles,
                       tmp.get(), s);
  k_level_totals<<<1, 32, 0, s>>>(counts.get(), offs.get(), ntiles, nl, totals.get());
  ADATM_LAUNCH();
  uint32_t host_tot[kMaxModes] = {0};
  ADATM_CUDA(cudaMemcpyAsync(host_tot, totals.get(), sizeof(uint32_t) * nl, cudaMemcpyDeviceToHost, s));
  ADATM_CUDA(cudaStreamSynchronize(s));
  for (int l = 0; l < nl; ++l) nfibs[l] = host_tot[l];
  nfibs[nl] = n;
}

// Close depths of level l's nodes from level l-1's: the last child of every
// parent p gets 1 + (close depth of p). Launched for l = 1..N-1 in order.
__global__ void k_close_depth(const uint32_t *fptr_parent, uint64_t nparent,
                              const uint8_t *cd_parent, uint8_t *cd_child) {
  const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nparent) return;
  const uint32_t last = fptr_parent[p + 1] - 1;
  cd_child[last] = (uint8_t)(1 + (cd_parent ? cd_parent[p] : 0));
}

void build_close_depths(DevCsf &out, cudaStream_t s) {
  const int N = out.nmodes;
  for (int l = 1; l < N; ++l) {
    const uint64_t n = l == N - 1 ? out.nnz : out.nfibs[l];
    out.cdepth[l].alloc(n);
    if (n == 0) continue;
    ADATM_CUDA(cudaMemsetAsync(out.cdepth[l].get(), 0, n, s));
    const uint64_t np = out.nfibs[l - 1];
    k_close_depth<<<(unsigned)((np + 255) / 256), 256, 0, s>>>(
        out.fptr[l - 1].get(), np, l >= 2 ? out.cdepth[l - 1].get() : nullptr,
        out.cdepth[l].get());
    ADATM_LAUNCH();
  }
}

template <int W>
void build_w(const DevCoo &coo, const uint64_t *perm, const KeySpec &spec, DevCsf &out,
             cudaStream_t s) {
  const uint64_t n = coo.nnz;
  const int N = coo.nmodes;
  SortBufs<W> b;
  sort_keys<W>(coo, perm, spec, b, s);
  DevBuf<uint32_t> offs;
  uint32_t ntiles = 0;
  count_levels<W>(b, n, spec, offs, ntiles, out.nfibs, s);
  LevelOut lo;
  for (int l = 0; l < kMaxModes; ++l) {
    lo.fptr[l] = nullptr;
    lo.fids[l] = nullptr;
  }
  for (int l = 0; l < N - 1; ++l) {
    out.fptr[l].alloc(out.nfibs[l] + 1);
    out.fids[l].alloc(out.nfibs[l]);
    lo.fptr[l] = out.fptr[l].get();
    lo.fids[l] = out.fids[l].get();
  }
  out.fids[N - 1].alloc(n);
  lo.fids[N - 1] = out.fids[N - 1].get();
  out.vals64.alloc(n);
  out.vals32.alloc(n);
  k_level_fill<W><<<ntiles, kLvThreads, 0, s>>>(b.keys, b.order, n, spec, offs.get(), ntiles, lo,
                                                coo.vals.get(), out.vals64.get(),
                                                out.vals32.get());
  ADATM_LAUNCH();
  DevBuf<uint32_t> totals(kMaxModes);
  uint32_t ht[kMaxModes] = {0};
  for (int l = 0; l < N - 1; ++l) ht[l] = (uint32_t)out.nfibs[l];
  ADATM_CUDA(cudaMemcpyAsync(totals.get(), ht, sizeof(ht), cudaMemcpyHostToDevice, s));
  k_level_tails<<<1, 32, 0, s>>>(lo, totals.get(), N - 1, n);
  ADATM_LAUNCH();
  build_close_depths(out, s);
  ADATM_CUDA(cudaStreamSynchronize(s));
}

template <int W>
void count_w(const DevCoo &coo, const uint64_t *perm, const KeySpec &spec, uint64_t *nfibs,
             cudaStream_t s) {
  SortBufs<W> b;
  sort_keys<W>(coo, perm, spec, b, s);
  DevBuf<uint32_t> offs;
  uint32_t ntiles = 0;
  count_levels<W>(b, coo.nnz, spec, offs, ntiles, nfibs, s);
}

// ---------------------------------------------------------------------------
// COO upload, clean-up and generation
// ---------------------------------------------------------------------------
__global__ void k_narrow(const uint64_t *in, uint32_t *out, uint64_t n, uint64_t dim,
                         unsigned int *bad) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t v = in[i];
  if (v >= dim) {
    atomicOr(bad, 1u);
    out[i] = 0;
  } else {
    out[i] = (uint32_t)v;
  }
}

template <int W>
__global__ void k_dedup(const Key<W> *keys, const uint32_t *order, uint64_t n,
                        const uint32_t *seg, KeySpec spec, const double *vals_in, IdxPtrs outp,
                        uint32_t **out_idx_unused, double *vals_out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Key<W> k = keys[i];
  if (i > 0 && key_equal<W>(k, keys[i - 1])) return;
  double sum = vals_in[order[i]];
  for (uint64_t j = i + 1; j < n; ++j) {
    if (!key_equal<W>(keys[j], k)) break;
    sum += vals_in[order[j]];
  }
  const uint32_t o = seg[i];
  vals_out[o] = sum;
  for (int l = 0; l < spec.nlev; ++l) const_cast<uint32_t *>(outp.p[l])[o] = key_field<W>(k, spec, l);
  (void)out_idx_unused;
}

template <int W>
__global__ void k_newkey_flags(const Key<W> *keys, uint64_t n, uint32_t *flags) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  flags[i] = (i == 0 || !key_equal<W>(keys[i], keys[i - 1])) ? 1u : 0u;
}

__global__ void k_mark_used(const uint32_t *idx, uint64_t n, uint32_t *used) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) used[idx[i]] = 1u;
}

__global__ void k_remap(uint32_t *idx, uint64_t n, const uint32_t *map) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) idx[i] = map[idx[i]];
}

template <int W>
void clean_w(const DevCoo &in, DevCoo &out, const KeySpec &spec, cudaStream_t s) {
  const uint64_t n = in.nnz;
  const int N = in.nmodes;
  uint64_t perm[kMaxModes];
  for (int m = 0; m < N; ++m) perm[m] = (uint64_t)m;
  SortBufs<W> b;
  sort_keys<W>(in, perm, spec, b, s);
  DevBuf<uint32_t> flags(n), seg(n), tmp(scan_tmp_words(n));
  const unsigned blocks = (unsigned)((n + 255) / 256);
  k_newkey_flags<W><<<blocks, 256, 0, s>>>(b.keys, n, flags.get());
  ADATM_LAUNCH();
  exclusive_scan_u32(flags.get(), seg.get(), n, tmp.get(), s);
  uint32_t last_seg = 0, last_flag = 0;
  ADATM_CUDA(cudaMemcpyAsync(&last_seg, seg.get() + n - 1, 4, cudaMemcpyDeviceToHost, s));
  ADATM_CUDA(cudaMemcpyAsync(&last_flag, flags.get() + n - 1, 4, cudaMemcpyDeviceToHost, s));
  ADATM_CUDA(cudaStreamSynchronize(s));
  const uint64_t nu = (uint64_t)last_seg + last_flag;
  out.nmodes = N;
  out.nnz = nu;
  IdxPtrs op;
  for (int l = 0; l < kMaxModes; ++l) op.p[l] = nullptr;
  for (int m = 0; m < N; ++m) {
    out.idx[m].alloc(nu);
    op.p[m] = out.idx[m].get();
  }
  out.vals.alloc(nu);
  k_dedup<W><<<blocks, 256, 0, s>>>(b.keys, b.order, n, seg.get(), spec, in.vals.get(), op, nullptr,
                                    out.vals.get());
  ADATM_LAUNCH();
  // compact empty slices of every mode
  for (int m = 0; m < N; ++m) {
    const uint64_t d = in.dims[m];
    DevBuf<uint32_t> used(d), map(d), mtmp(scan_tmp_words(d));
    ADATM_CUDA(cudaMemsetAsync(used.get(), 0, d * sizeof(uint32_t), s));
    const unsigned ub = (unsigned)((nu + 255) / 256);
    k_mark_used<<<ub, 256, 0, s>>>(out.idx[m].get(), nu, used.get());
    ADATM_LAUNCH();
    exclusive_scan_u32(used.get(), map.get(), d, mtmp.get(), s);
    uint32_t lm = 0, lu = 0;
    ADATM_CUDA(cudaMemcpyAsync(&lm, map.get() + d - 1, 4, cudaMemcpyDeviceToHost, s));
    ADATM_CUDA(cudaMemcpyAsync(&lu, used.get() + d - 1, 4, cudaMemcpyDeviceToHost, s));
    k_remap<<<ub, 256, 0, s>>>(out.idx[m].get(), nu, map.get());
    ADATM_LAUNCH();
    ADATM_CUDA(cudaStreamSynchronize(s));
    out.dims[m] = (uint64_t)lm + lu;
  }
}

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double u01(uint64_t x) {
  return (double)(x >> 11) * (1.0 / 9007199254740992.0);
}

struct GenArgs {
  uint32_t *idx[kMaxModes];
  const double *cdf[kMaxModes];  // nullptr = uniform
  uint64_t dims[kMaxModes];
  uint64_t key[kMaxModes + 2];
  int nmodes;
  int value_kind;
  double mu, sigma;
};

__global__ void k_generate(GenArgs a, uint64_t n, double *vals) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int m = 0; m < a.nmodes; ++m) {
    const double u = u01(mix64(a.key[m] + i));
    uint64_t k;
    if (a.cdf[m] == nullptr) {
      k = (uint64_t)(u * (double)a.dims[m]);
      if (k >= a.dims[m]) k = a.dims[m] - 1;
    } else {
      uint64_t lo = 0, hi = a.dims[m] - 1;  // smallest k with u < cdf[k]
      while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (u < a.cdf[m][mid])
          hi = mid;
        else
          lo = mid + 1;
      }
      k = lo;
    }
    a.idx[m][i] = (uint32_t)k;
  }
  const double u1 = u01(mix64(a.key[a.nmodes] + i));
  if (a.value_kind == 0) {
    vals[i] = u1;
  } else {
    const double u2 = u01(mix64(a.key[a.nmodes + 1] + i));
    const double z = sqrt(-2.0 * log(1.0 - u1)) * cospi(2.0 * u2);
    vals[i] = exp(a.mu + a.sigma * z);
  }
}

__global__ void k_widen(const uint32_t *in, uint64_t *out, uint64_t n) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i];
}

}  // namespace

// ---------------------------------------------------------------------------
// public entry points
// ---------------------------------------------------------------------------
void coo_upload(DevCoo &out, int nmodes, uint64_t nnz, const uint64_t *dims,
                const uint64_t *const *inds, const double *vals, cudaStream_t s) {
  if (nmodes < 3 || nmodes > kMaxModes) throw BadInput("tensor order must be 3..8");
  if (nnz >= 0xFFFFFFFFull) throw BadInput("nnz must be below 2^32-1");
  out.nmodes = nmodes;
  out.nnz = nnz;
  DevBuf<uint64_t> tmp(nnz);
  DevBuf<unsigned int> bad(1);
  ADATM_CUDA(cudaMemsetAsync(bad.get(), 0, sizeof(unsigned int), s));
  for (int m = 0; m < nmodes; ++m) {
    if (dims[m] == 0 || dims[m] >= 0xFFFFFFFFull) throw BadInput("dimension out of range");
    out.dims[m] = dims[m];
    out.idx[m].alloc(nnz);
    if (nnz == 0) continue;
    ADATM_CUDA(cudaMemcpyAsync(tmp.get(), inds[m], nnz * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
    k_narrow<<<(unsigned)((nnz + 255) / 256), 256, 0, s>>>(tmp.get(), out.idx[m].get(), nnz,
                                                           dims[m], bad.get());
    ADATM_LAUNCH();
  }
  out.vals.alloc(nnz);
  if (nnz)
    ADATM_CUDA(cudaMemcpyAsync(out.vals.get(), vals, nnz * sizeof(double), cudaMemcpyHostToDevice, s));
  unsigned int hb = 0;
  ADATM_CUDA(cudaMemcpyAsync(&hb, bad.get(), sizeof(hb), cudaMemcpyDeviceToHost, s));
  ADATM_CUDA(cudaStreamSynchronize(s));
  if (hb) throw BadInput("a coordinate is outside its dimension");
}

void coo_clean(const DevCoo &in, DevCoo &out, cudaStream_t s) {
  if (in.nnz == 0) {
    out.nmodes = in.nmodes;
    out.nnz = 0;
    for (int m = 0; m < in.nmodes; ++m) out.dims[m] = 0;
    return;
  }
  uint64_t perm[kMaxModes];
  for (int m = 0; m < in.nmodes; ++m) perm[m] = (uint64_t)m;
  const KeySpec spec = make_key_spec(in.nmodes, in.dims, perm);
  switch (spec.words) {
    case 1: clean_w<1>(in, out, spec, s); break;
    case 2: clean_w<2>(in, out, spec, s); break;
    default: clean_w<3>(in, out, spec, s); break;
  }
}

void coo_generate(DevCoo &out, int nmodes, const uint64_t *dims, uint64_t nnz,
                  const double *alpha, int value_kind, double mu, double sigma, uint64_t seed,
                  cudaStream_t s) {
  if (nmodes < 3 || nmodes > kMaxModes) throw BadInput("tensor order must be 3..8");
  out.nmodes = nmodes;
  out.nnz = nnz;
  GenArgs a;
  a.nmodes = nmodes;
  a.value_kind = value_kind;
  a.mu = mu;
  a.sigma = sigma;
  std::vector<DevBuf<double>> cdfs(nmodes);
  for (int m = 0; m < kMaxModes; ++m) {
    a.idx[m] = nullptr;
    a.cdf[m] = nullptr;
    a.dims[m] = 0;
  }
  auto hmix = [](uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  for (int m = 0; m < nmodes + 2; ++m) a.key[m] = hmix(seed * 0x100000001B3ull + 0x1000u + (uint64_t)m);
  for (int m = 0; m < nmodes; ++m) {
    out.dims[m] = dims[m];
    a.dims[m] = dims[m];
    out.idx[m].alloc(nnz);
    a.idx[m] = out.idx[m].get();
    if (alpha && alpha[m] > 0) {
      std::vector<double> c(dims[m]);
      double acc = 0;
      for (uint64_t k = 0; k < dims[m]; ++k) {
        acc += std::pow((double)(k + 1), -alpha[m]);
        c[k] = acc;
      }
      for (uint64_t k = 0; k < dims[m]; ++k) c[k] /= acc;
      c[dims[m] - 1] = 1.0;
      cdfs[m].alloc(dims[m]);
      ADATM_CUDA(cudaMemcpyAsync(cdfs[m].get(), c.data(), dims[m] * sizeof(double),
                                 cudaMemcpyHostToDevice, s));
      a.cdf[m] = cdfs[m].get();
      ADATM_CUDA(cudaStreamSynchronize(s));
    }
  }
  out.vals.alloc(nnz);
  if (nnz) {
    k_generate<<<(unsigned)((nnz + 255) / 256), 256, 0, s>>>(a, nnz, out.vals.get());
    ADATM_LAUNCH();
  }
  ADATM_CUDA(cudaStreamSynchronize(s));
}

void csf_build(const DevCoo &coo, const uint64_t *perm, DevCsf &out, cudaStream_t s) {
  const int N = coo.nmodes;
  out.nmodes = N;
  out.nnz = coo.nnz;
  for (int m = 0; m < N; ++m) {
    out.dims[m] = coo.dims[m];
    out.dim_perm[m] = perm[m];
  }
  if (coo.nnz == 0) {
    for (int l = 0; l < N - 1; ++l) {
      out.nfibs[l] = 0;
      out.fptr[l].alloc(1);
      ADATM_CUDA(cudaMemsetAsync(out.fptr[l].get(), 0, sizeof(uint32_t), s));
    }
    out.nfibs[N - 1] = 0;
    ADATM_CUDA(cudaStreamSynchronize(s));
    return;
  }
  const KeySpec spec = make_key_spec(N, coo.dims, perm);
  switch (spec.words) {
    case 1: build_w<1>(coo, perm, spec, out, s); break;
    case 2: build_w<2>(coo, perm, spec, out, s); break;
    default: build_w<3>(coo, perm, spec, out, s); break;
  }
}

void csf_count(const DevCoo &coo, const uint64_t *perm, uint64_t *nfibs, cudaStream_t s) {
  const int N = coo.nmodes;
  if (coo.nnz == 0) {
    for (int l = 0; l < N; ++l) nfibs[l] = 0;
    return;
  }
  const KeySpec spec = make_key_spec(N, coo.dims, perm);
  switch (spec.words) {
    case 1: count_w<1>(coo, perm, spec, nfibs, s); break;
    case 2: count_w<2>(coo, perm, spec, nfibs, s); break;
    default: count_w<3>(coo, perm, spec, nfibs, s); break;
  }
}

void csf_download(const DevCsf &c, HostCsfArrays &h, cudaStream_t s) {
  const int N = c.nmodes;
  h.fptr.assign(N, {});
  h.fids.assign(N, {});
  uint64_t maxn = 1;
  for (int l = 0; l < N; ++l) maxn = std::max<uint64_t>(maxn, c.nfibs[l] + 1);
  DevBuf<uint64_t> wide(maxn);
  auto pull = [&](const DevBuf<uint32_t> &src, uint64_t n, std::vector<uint64_t> &dst) {
    dst.assign(n, 0);
    if (n == 0 || src.get() == nullptr) return;
    k_widen<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src.get(), wide.get(), n);
    ADATM_LAUNCH();
    ADATM_CUDA(cudaMemcpyAsync(dst.data(), wide.get(), n * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    ADATM_CUDA(cudaStreamSynchronize(s));
  };
  for (int l = 0; l < N; ++l) {
    if (l < N - 1) pull(c.fptr[l], c.nfibs[l] + 1, h.fptr[l]);
    pull(c.fids[l], c.nfibs[l], h.fids[l]);
  }
  h.vals.assign(c.nnz, 0.0);
  if (c.nnz)
    ADATM_CUDA(cudaMemcpyAsync(h.vals.data(), c.vals64.get(), c.nnz * sizeof(double),
                               cudaMemcpyDeviceToHost, s));
  ADATM_CUDA(cudaStreamSynchronize(s));
}

}  // namespace adatm
