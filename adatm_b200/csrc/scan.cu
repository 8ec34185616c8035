// scan.cu -- exclusive prefix sums on the device, in three launches without
// any inter-block waiting: per-tile sums, one block scanning the tile sums,
// per-tile scans that add their tile offset.
#include "common.cuh"

namespace adatm {

namespace {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Block-wide exclusive scan of one value per thread; returns the exclusive
// prefix and writes the block total to *total.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t *total) {
  __shared__ uint32_t warp_sums[kScanThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = warp_incl_scan(v);
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kScanThreads / 32 ? warp_sums[lane] : 0;
    uint32_t wi = warp_incl_scan(w);
    if (lane < kScanThreads / 32) warp_sums[lane] = wi - w;
    if (lane == kScanThreads / 32 - 1) *total = wi;
  }
  __syncthreads();
  uint32_t r = warp_sums[warp] + incl - v;
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const uint32_t *in, size_t n,
                                                              uint32_t *tile_sums) {
  const size_t base = (size_t)blockIdx.x * kScanTile;
  uint32_t s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    size_t idx = base + (size_t)i * kScanThreads + threadIdx.x;
    if (idx < n) s += in[idx];
  }
  __shared__ uint32_t tot;
  block_excl_scan(s, &tot);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

// One block: exclusive scan of `n` values in place, chunk by chunk.
__global__ void __launch_bounds__(kScanThreads) k_scan_single(uint32_t *data, size_t n) {
  __shared__ uint32_t tot;
  uint32_t carry = 0;
  for (size_t base = 0; base < n; base += kScanTile) {
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
      size_t idx = base + (size_t)threadIdx.x * kScanItems + i;
      v[i] = idx < n ? data[idx] : 0;
      s += v[i];
    }
    uint32_t ex = block_excl_scan(s, &tot) + carry;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
      size_t idx = base + (size_t)threadIdx.x * kScanItems + i;
      if (idx < n) data[idx] = ex;
      ex += v[i];
    }
    carry += tot;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_final(const uint32_t *in, uint32_t *out,
                                                             size_t n, const uint32_t *tile_off) {
  const size_t base = (size_t)blockIdx.x * kScanTile;
  uint32_t v[kScanItems];
  uint32_t s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    size_t idx = base + (size_t)threadIdx.x * kScanItems + i;
    v[i] = idx < n ? in[idx] : 0;
    s += v[i];
  }
  __shared__ uint32_t tot;
  uint32_t ex = block_excl_scan(s, &tot) + tile_off[blockIdx.x];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    size_t idx = base + (size_t)threadIdx.x * kScanItems + i;
    if (idx < n) out[idx] = ex;
    ex += v[i];
  }
}

}  // namespace

size_t scan_tmp_words(size_t n) { return (n + kScanTile - 1) / kScanTile + 1; }

void exclusive_scan_u32(const uint32_t *in, uint32_t *out, size_t n, uint32_t *tmp,
                        cudaStream_t stream) {
  if (n == 0) return;
  const size_t tiles = (n + kScanTile - 1) / kScanTile;
  k_scan_reduce<<<(unsigned)tiles, kScanThreads, 0, stream>>>(in, n, tmp);
  ADATM_LAUNCH();
  k_scan_single<<<1, kScanThreads, 0, stream>>>(tmp, tiles);
  ADATM_LAUNCH();
  k_scan_final<<<(unsigned)tiles, kScanThreads, 0, stream>>>(in, out, n, tmp);
  ADATM_LAUNCH();
}

}  // namespace adatm
