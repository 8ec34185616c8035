// als.cu -- dense CP-ALS kernels (see als.cuh).
#include <algorithm>
#include <mutex>

#include "als.cuh"

namespace adatm {

namespace {
void set_attributes();
}

void AlsWork::init(int nmodes_, int R_, int nblocks_, int max_iters) {
  nmodes = nmodes_;
  R = R_;
  ldr = ldr_of(R_);
  nblocks = nblocks_;
  vinv64.alloc((size_t)R * R);
  part_gram.alloc((size_t)nblocks * R * R);
  part_max.alloc((size_t)nblocks * R);
  part_inner.alloc((size_t)nblocks * R);
  lambda.alloc(R);
  scalars.alloc(8);
  iter.alloc(1);
  max_trace = std::max(1, max_iters);
  fit_trace.alloc(max_trace);
  ADATM_CUDA(cudaMemset(scalars.get(), 0, 8 * sizeof(double)));
  ADATM_CUDA(cudaMemset(iter.get(), 0, sizeof(int)));
  ADATM_CUDA(cudaMemset(fit_trace.get(), 0, max_trace * sizeof(double)));
  set_attributes();
}

namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__global__ void k_factor_init(float *A, __nv_bfloat16 *Ab, uint64_t rows, int R, int ldr,
                              uint64_t key) {
  const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= rows * (uint64_t)ldr) return;
  const uint64_t i = e / ldr;
  const int r = (int)(e % ldr);
  float v = 0.f;
  if (r < R) {
    const uint64_t x = i * (uint64_t)R + r;
    v = (float)((double)(mix64(key + x) >> 11) * (1.0 / 9007199254740992.0));
  }
  if (Ab) {
    // BF16 factors: the rounded value is the factor (see to_bf16)
    const __nv_bfloat16 b = __float2bfloat16(v);
    Ab[e] = b;
    v = __bfloat162float(b);
  }
  A[e] = v;
}

__global__ void k_to_bf16(float *A, __nv_bfloat16 *Ab, uint64_t n) {
  const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) {
    const __nv_bfloat16 b = __float2bfloat16(A[e]);
    Ab[e] = b;
    A[e] = __bfloat162float(b);
  }
}

constexpr int kFrobThreads = 256;

__global__ void k_frob_partial(const double *v, uint64_t n, double *part) {
  double s = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    s += v[i] * v[i];
  __shared__ double red[kFrobThreads];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = kFrobThreads / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void k_frob_final(const double *part, int n, double *out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0;
    for (int i = 0; i < n; ++i) s += part[i];
    out[0] = s;
  }
}

// ---------------------------------------------------------------------------
// Gram Hadamard + inverse, one block. V = Hadamard of every G[m], m != mode,
// is symmetric positive definite, so Gauss-Jordan elimination in place needs
// no pivoting (each pivot is a diagonal entry of a Schur complement of V,
// hence positive). All R steps stay in shared memory.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_gram_inverse(GramSet g, int nmodes, int mode, int R,
                                                      double *X) {
  extern __shared__ double V[];  // R x R, then the pivot column (R)
  double *col = V + R * R;
  const int tid = threadIdx.x;
  for (int e = tid; e < R * R; e += blockDim.x) {
    double v = 1.0;
    for (int m = 0; m < nmodes; ++m)
      if (m != mode) v *= g.G[m][e];
    V[e] = v;
  }
  __syncthreads();
  for (int j = 0; j < R; ++j) {
    const double p = V[j * R + j];
    for (int i = tid; i < R; i += blockDim.x) col[i] = V[i * R + j];
    __syncthreads();
    // pivot row: V[j][k] = (k == j ? 1 : V[j][k]) / p
    for (int k = tid; k < R; k += blockDim.x) V[j * R + k] = (k == j ? 1.0 : V[j * R + k]) / p;
    __syncthreads();
    // other rows: V[i][k] = (k == j ? 0 : V[i][k]) - col[i] * V[j][k]
    for (int e = tid; e < R * R; e += blockDim.x) {
      const int i = e / R, k = e % R;
      if (i == j) continue;
      V[e] = (k == j ? 0.0 : V[e]) - col[i] * V[j * R + k];
    }
    __syncthreads();
  }
  for (int e = tid; e < R * R; e += blockDim.x) {
    // symmetrise: the two triangles differ only by rounding
    const int i = e / R, k = e % R;
    const double v = 0.5 * (V[e] + V[k * R + i]);
    X[e] = v;
  }
}

// ---------------------------------------------------------------------------
// Row update A_raw = M * Vinv (or A_raw = M when vinv == nullptr), with
// per-block FP64 partial Gram and column maxima of A_raw.
// ---------------------------------------------------------------------------
struct UpdArgs {
  int split;           // Gram products as 3 TF32 terms (FP32 rows) or 1 (BF16-valued rows)
  const double *Md;    // MTTKRP rows (FP64) of an update, or nullptr
  const float *M;      // rows whose Gram alone is wanted (vinv == nullptr)
  const double *vinv;  // R x R fp64, or nullptr for identity
  float *A;           // output rows (may alias M when vinv == nullptr)
  uint64_t rows;
  int R, ldr;
  double *part_gram;  // gridDim x R x R
  double *part_max;   // gridDim x R
};

// One m16n8k8 TF32 tensor-core product with FP32 accumulation, c += a * b
// (A 16 x 8 row-major, B 8 x 8 column-major, per-thread fragments of the
// warp-wide tiles).
__device__ __forceinline__ void mma_tf32(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return r;
}

// Row pass of a mode update (or of a plain Gram). Each block takes row
// groups of 256 / LANES rows; the rows (A = M V^-1, or M itself) are staged
// in shared memory and their Gram X^T X is taken on the tensor cores: G is
// tiled in 16 x 8 tiles spread over the block's 8 warps; every 8 rows of a
// tile are one m16n8k8 TF32 MMA step with FP32 accumulation, added to FP64
// per-thread sums after the step. FP32 rows split into a TF32 big
// part and a TF32 remainder, and big*big + big*rem + rem*big keeps the
// products to ~2^-22 (split = 1); BF16-valued rows are exact in TF32 and
// take one product.
template <int LANES>
__global__ void __launch_bounds__(256) k_update(UpdArgs a) {
  constexpr int GROUPS = 256 / LANES;
  constexpr int RMAX = 4 * LANES;
  constexpr int RS = RMAX + 8;          // staged row stride (bank-conflict free MMA loads)
  constexpr int TN = RMAX / 8;          // 8-column tiles of G
  constexpr int NT = (RMAX / 16) * TN;  // 16 x 8 tiles
  constexpr int TPW = (NT + 7) / 8;     // tiles per warp
  extern __shared__ double usm[];
  double *vinv = usm;                                            // RMAX x RMAX
  float *rowbuf = reinterpret_cast<float *>(usm + RMAX * RMAX);  // GROUPS x RS
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31, gid = lane >> 2, tig = lane & 3;
  const int g = tid / LANES, t = tid % LANES, col = 4 * t;
  const int R = a.R;
  const bool act = col < R;
  const unsigned gmask =
      LANES == 32 ? 0xffffffffu : (((1u << LANES) - 1u) << ((tid & 31) / LANES * LANES));
  if (a.vinv) {
    for (int e = tid; e < RMAX * RMAX; e += 256) {
      const int k = e / RMAX, c = e % RMAX;
      vinv[e] = (k < R && c < R) ? a.vinv[k * R + c] : 0.0;
    }
  }
  double gacc[TPW][4];
#pragma unroll
  for (int tt = 0; tt < TPW; ++tt)
#pragma unroll
    for (int q = 0; q < 4; ++q) gacc[tt][q] = 0.0;
  double cmax = 0.0;
  __syncthreads();
  const int kq = (R + 3) / 4;
  for (uint64_t row0 = (uint64_t)blockIdx.x * GROUPS; row0 < a.rows;
       row0 += (uint64_t)gridDim.x * GROUPS) {
    const uint64_t i = row0 + g;
    const bool valid = i < a.rows;
    double md[4] = {0.0, 0.0, 0.0, 0.0};
    if (valid && act) {
      if (a.Md) {
        const double2 lo = *reinterpret_cast<const double2 *>(a.Md + i * a.ldr + col);
        const double2 hi = *reinterpret_cast<const double2 *>(a.Md + i * a.ldr + col + 2);
        md[0] = lo.x;
        md[1] = lo.y;
        md[2] = hi.x;
        md[3] = hi.y;
      } else {
        const float4 f = *reinterpret_cast<const float4 *>(a.M + i * a.ldr + col);
        md[0] = f.x;
        md[1] = f.y;
        md[2] = f.z;
        md[3] = f.w;
      }
    }
    float4 o;
    if (a.vinv) {
      // A = M V^-1 with V^-1 and the sums in FP64: V (the Hadamard of the
      // other modes' Grams) is often ill-conditioned, and FP32 sums of its
      // inverse's large entries of both signs lose the fit's digits
      double o0 = 0.0, o1 = 0.0, o2 = 0.0, o3 = 0.0;
      for (int kk = 0; kk < kq; ++kk) {
        const double m4[4] = {__shfl_sync(gmask, md[0], kk, LANES), __shfl_sync(gmask, md[1], kk, LANES),
                              __shfl_sync(gmask, md[2], kk, LANES), __shfl_sync(gmask, md[3], kk, LANES)};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const double *vr = vinv + (4 * kk + q) * RMAX + col;
          const double2 lo = *reinterpret_cast<const double2 *>(vr);
          const double2 hi = *reinterpret_cast<const double2 *>(vr + 2);
          o0 = fma(m4[q], lo.x, o0);
          o1 = fma(m4[q], lo.y, o1);
          o2 = fma(m4[q], hi.x, o2);
          o3 = fma(m4[q], hi.y, o3);
        }
      }
      o = make_float4((float)o0, (float)o1, (float)o2, (float)o3);
      if (valid && act) *reinterpret_cast<float4 *>(a.A + i * a.ldr + col) = o;
    } else {
      o = make_float4((float)md[0], (float)md[1], (float)md[2], (float)md[3]);
    }
    *reinterpret_cast<float4 *>(rowbuf + g * RS + col) =
        valid ? o : make_float4(0.f, 0.f, 0.f, 0.f);
    __syncthreads();
#pragma unroll
    for (int tt = 0; tt < TPW; ++tt) {
      const int tile = warp + 8 * tt;
      const int i0 = (tile / TN) * 16, j0 = (tile % TN) * 8;
      if (tile < NT && i0 < R && j0 < R) {
#pragma unroll
        for (int k0 = 0; k0 < GROUPS; k0 += 8) {
          float c[4] = {0.f, 0.f, 0.f, 0.f};
          // A = X^T (rows i0.., the group's rows as k), B = X (columns j0..)
          const float *x0 = rowbuf + (k0 + tig) * RS, *x1 = rowbuf + (k0 + tig + 4) * RS;
          const float av[4] = {x0[i0 + gid], x0[i0 + gid + 8], x1[i0 + gid], x1[i0 + gid + 8]};
          const float bv[2] = {x0[j0 + gid], x1[j0 + gid]};
          uint32_t ab[4], bb[2];
#pragma unroll
          for (int q = 0; q < 4; ++q) ab[q] = to_tf32(av[q]);
          bb[0] = to_tf32(bv[0]);
          bb[1] = to_tf32(bv[1]);
          mma_tf32(c, ab, bb);
          if (a.split) {
            uint32_t as[4], bs[2];
#pragma unroll
            for (int q = 0; q < 4; ++q) as[q] = to_tf32(av[q] - __uint_as_float(ab[q]));
            bs[0] = to_tf32(bv[0] - __uint_as_float(bb[0]));
            bs[1] = to_tf32(bv[1] - __uint_as_float(bb[1]));
            mma_tf32(c, ab, bs);
            mma_tf32(c, as, bb);
          }
#pragma unroll
          for (int q = 0; q < 4; ++q) gacc[tt][q] += (double)c[q];
        }
      }
    }
    if (tid < R)
      for (int gi = 0; gi < GROUPS; ++gi) cmax = fmax(cmax, (double)rowbuf[gi * RS + tid]);
    __syncthreads();
  }
#pragma unroll
  for (int tt = 0; tt < TPW; ++tt) {
    const int tile = warp + 8 * tt;
    const int i0 = (tile / TN) * 16, j0 = (tile % TN) * 8;
    if (tile >= NT || i0 >= R || j0 >= R) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = i0 + gid + (q >= 2 ? 8 : 0), j = j0 + 2 * tig + (q & 1);
      if (i < R && j < R) a.part_gram[(size_t)blockIdx.x * R * R + i * R + j] = gacc[tt][q];
    }
  }
  if (tid < R) a.part_max[(size_t)blockIdx.x * R + tid] = cmax;
}

// Sum the partial Grams; with lam != nullptr also derive lambda (2-norm on the
// first iteration, max-norm floored at 1 after) and scale G by 1/(l_r l_s).
// Grid: ceil(R*R / kFinEntries) blocks of 256 threads; a block sums
// kFinEntries entries, its 256 / kFinEntries warps splitting the partials, so
// no thread walks a long chain of dependent L2 loads. Every block derives the
// lambda values it needs; block 0 stores them.
constexpr int kFinEntries = 32;
constexpr int kFinParts = 256 / kFinEntries;

__global__ void __launch_bounds__(256) k_finalize(const double *part_gram, const double *part_max,
                                                  int nblocks, int R, double *G, double *lam,
                                                  const int *iter) {
  __shared__ double slam[128];
  __shared__ double red[256];
  const int tid = threadIdx.x;
  if (lam) {
    const bool first = (iter == nullptr) || (*iter == 0);
    const int parts = 256 / R;  // R <= 128
    const int r = tid % R, q = tid / R;
    double v = 0.0;
    if (q < parts) {
      if (first) {
        for (int b = q; b < nblocks; b += parts) v += part_gram[(size_t)b * R * R + r * R + r];
      } else {
        for (int b = q; b < nblocks; b += parts) v = fmax(v, part_max[(size_t)b * R + r]);
      }
    }
    red[tid] = v;
    __syncthreads();
    if (tid < R) {
      double a = 0.0;
      for (int k = 0; k < parts; ++k) a = first ? a + red[k * R + tid] : fmax(a, red[k * R + tid]);
      const double l = first ? sqrt(a) : fmax(a, 1.0);
      slam[tid] = l;
      if (blockIdx.x == 0) lam[tid] = l;
    }
    __syncthreads();
  }
  const int e = blockIdx.x * kFinEntries + tid % kFinEntries;
  const int q = tid / kFinEntries;
  double acc = 0.0;
  if (e < R * R)
    for (int b = q; b < nblocks; b += kFinParts) acc += part_gram[(size_t)b * R * R + e];
  red[tid] = acc;
  __syncthreads();
  if (tid < kFinEntries && e < R * R) {
    double sum = 0.0;
    for (int k = 0; k < kFinParts; ++k) sum += red[k * kFinEntries + tid];
    if (lam) sum /= slam[e / R] * slam[e % R];
    G[e] = sum;
  }
}

int finalize_blocks(int R) { return (R * R + kFinEntries - 1) / kFinEntries; }

// A /= lambda (fp32), bf16 copy, optional partial <A, M> per column.
template <int LANES>
__global__ void __launch_bounds__(256) k_scale(float *A, __nv_bfloat16 *Ab, const double *M,
                                               uint64_t rows, int R, int ldr, const double *lam,
                                               double *part_inner) {
  constexpr int GROUPS = 256 / LANES;
  const int tid = threadIdx.x;
  const int g = tid / LANES, t = tid % LANES, col = 4 * t;
  const bool act = col < R;
  float4 il = make_float4(0.f, 0.f, 0.f, 0.f);
  if (act) {
    il.x = col + 0 < R ? (float)(1.0 / lam[col + 0]) : 0.f;
    il.y = col + 1 < R ? (float)(1.0 / lam[col + 1]) : 0.f;
    il.z = col + 2 < R ? (float)(1.0 / lam[col + 2]) : 0.f;
    il.w = col + 3 < R ? (float)(1.0 / lam[col + 3]) : 0.f;
  }
  double in0 = 0, in1 = 0, in2 = 0, in3 = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * GROUPS + g; i < rows; i += (uint64_t)gridDim.x * GROUPS) {
    if (!act) continue;
    float4 v = *reinterpret_cast<float4 *>(A + i * ldr + col);
    v.x *= il.x;
    v.y *= il.y;
    v.z *= il.z;
    v.w *= il.w;
    if (Ab) {
      // BF16 factors: the rounded row replaces the FP32 row too, so the
      // Gram, the MTTKRPs and the fit all see the same factor
      __nv_bfloat162 lo = __floats2bfloat162_rn(v.x, v.y);
      __nv_bfloat162 hi = __floats2bfloat162_rn(v.z, v.w);
      uint2 raw;
      raw.x = *reinterpret_cast<uint32_t *>(&lo);
      raw.y = *reinterpret_cast<uint32_t *>(&hi);
      *reinterpret_cast<uint2 *>(Ab + i * ldr + col) = raw;
      const float2 flo = __bfloat1622float2(lo), fhi = __bfloat1622float2(hi);
      v = make_float4(flo.x, flo.y, fhi.x, fhi.y);
    }
    *reinterpret_cast<float4 *>(A + i * ldr + col) = v;
    if (part_inner) {
      const double2 lo = *reinterpret_cast<const double2 *>(M + i * ldr + col);
      const double2 hi = *reinterpret_cast<const double2 *>(M + i * ldr + col + 2);
      in0 += (double)v.x * lo.x;
      in1 += (double)v.y * lo.y;
      in2 += (double)v.z * hi.x;
      in3 += (double)v.w * hi.y;
    }
  }
  if (part_inner) {
    __shared__ double red[256 * 4];
    red[tid * 4 + 0] = in0;
    red[tid * 4 + 1] = in1;
    red[tid * 4 + 2] = in2;
    red[tid * 4 + 3] = in3;
    __syncthreads();
    if (tid < 4 * LANES) {
      const int tt = tid / 4, c = tid % 4;
      double s = 0;
      for (int gi = 0; gi < GROUPS; ++gi) s += red[(gi * LANES + tt) * 4 + c];
      const int column = 4 * tt + c;
      if (column < R) part_inner[(size_t)blockIdx.x * R + column] = s;
    }
  }
}

__global__ void k_fit(GramSet g, int nmodes, int R, const double *lam, const double *part_inner,
                      int nblocks, double *scalars, double *trace, int max_trace, int *iter) {
  __shared__ double red[256];
  const int tid = threadIdx.x;
  double nrm = 0;
  for (int e = tid; e < R * R; e += blockDim.x) {
    double h = 1.0;
    for (int m = 0; m < nmodes; ++m) h *= g.G[m][e];
    nrm += h * lam[e / R] * lam[e % R];
  }
  // <X, Z> = sum_r lam_r sum_b part_inner[b][r]: 256 / R threads per column
  double inner = 0;
  {
    const int parts = 256 / R, r = tid % R, q = tid / R;
    if (q < parts) {
      for (int b = q; b < nblocks; b += parts) inner += part_inner[(size_t)b * R + r];
      inner *= lam[r];
    }
  }
  red[tid] = nrm;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (tid < o) red[tid] += red[tid + o];
    __syncthreads();
  }
  const double norm = fabs(red[0]);
  __syncthreads();
  red[tid] = inner;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (tid < o) red[tid] += red[tid + o];
    __syncthreads();
  }
  if (tid == 0) {
    const double in = red[0];
    const double ttn = scalars[0];
    const double fit = 1.0 - sqrt(ttn + norm - 2.0 * in) / sqrt(ttn);
    scalars[1] = fit;
    scalars[2] = norm;
    scalars[3] = in;
    const int it = *iter;
    if (it < max_trace) trace[it] = fit;
    *iter = it + 1;
  }
}

int lanes_for(int R) {
  if (R <= 16) return 4;
  if (R <= 32) return 8;
  if (R <= 64) return 16;
  if (R <= 128) return 32;
  throw BadInput("rank above 128 is not supported by the GPU kernels");
}

template <int LANES>
constexpr size_t update_smem() {
  return (size_t)(4 * LANES * 4 * LANES) * sizeof(double) +
         (size_t)((256 / LANES) * (4 * LANES + 8)) * sizeof(float);
}

template <int LANES>
void launch_update(const UpdArgs &u, int nblocks, cudaStream_t s) {
  k_update<LANES><<<nblocks, 256, update_smem<LANES>(), s>>>(u);
  ADATM_LAUNCH();
}

// Kernels with more than 48 KB of dynamic shared memory must be opted in
// once, before any stream capture.
void set_attributes() {
  ADATM_CUDA(cudaFuncSetAttribute(k_update<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)update_smem<4>()));
  ADATM_CUDA(cudaFuncSetAttribute(k_update<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)update_smem<8>()));
  ADATM_CUDA(cudaFuncSetAttribute(k_update<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)update_smem<16>()));
  ADATM_CUDA(cudaFuncSetAttribute(k_update<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)update_smem<32>()));
  ADATM_CUDA(cudaFuncSetAttribute(k_gram_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (128 * 128 + 128) * (int)sizeof(double)));
}

// Row blocks of the update: enough to give every block at least one full
// batch of rows, at most the workspace's partial slots.
int update_blocks(uint64_t rows, int R, int max_blocks) {
  const uint64_t groups = 256 / lanes_for(R);
  const uint64_t need = (rows + groups - 1) / groups;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)max_blocks, need));
}

void run_update(const UpdArgs &u, int nblocks, cudaStream_t s) {
  switch (lanes_for(u.R)) {
    case 4: launch_update<4>(u, nblocks, s); break;
    case 8: launch_update<8>(u, nblocks, s); break;
    case 16: launch_update<16>(u, nblocks, s); break;
    default: launch_update<32>(u, nblocks, s); break;
  }
}

}  // namespace

void factor_init_device(float *A, __nv_bfloat16 *Ab, uint64_t rows, int R, int ldr, uint64_t seed,
                        uint64_t mode, cudaStream_t s) {
  auto hmix = [](uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  const uint64_t key = hmix(seed * 0x100000001B3ull + mode);
  const uint64_t n = rows * (uint64_t)ldr;
  if (n == 0) return;
  k_factor_init<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(A, Ab, rows, R, ldr, key);
  ADATM_LAUNCH();
}

void to_bf16(float *A, __nv_bfloat16 *Ab, uint64_t rows, int ldr, cudaStream_t s) {
  const uint64_t n = rows * (uint64_t)ldr;
  if (n == 0) return;
  k_to_bf16<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(A, Ab, n);
  ADATM_LAUNCH();
}

void gram(const float *A, uint64_t rows, int R, int ldr, double *G, AlsWork &w, cudaStream_t s,
          bool bf16_rows) {
  UpdArgs u;
  u.split = bf16_rows ? 0 : 1;
  u.Md = nullptr;
  u.M = A;
  u.vinv = nullptr;
  u.A = nullptr;
  u.rows = rows;
  u.R = R;
  u.ldr = ldr;
  u.part_gram = w.part_gram.get();
  u.part_max = w.part_max.get();
  const int nb = update_blocks(rows, R, w.nblocks);
  run_update(u, nb, s);
  k_finalize<<<finalize_blocks(R), 256, 0, s>>>(w.part_gram.get(), w.part_max.get(), nb, R, G, nullptr,
                               nullptr);
  ADATM_LAUNCH();
}

void frob_sq(const double *vals, uint64_t n, AlsWork &w, cudaStream_t s) {
  const int blocks = 256;
  if (w.frob_part.n < (size_t)blocks) w.frob_part.alloc(blocks);
  k_frob_partial<<<blocks, kFrobThreads, 0, s>>>(vals, n, w.frob_part.get());
  ADATM_LAUNCH();
  k_frob_final<<<1, 32, 0, s>>>(w.frob_part.get(), blocks, w.scalars.get());
  ADATM_LAUNCH();
  ADATM_CUDA(cudaStreamSynchronize(s));
}

void gram_inverse(const GramSet &g, int mode, AlsWork &w, cudaStream_t s) {
  const size_t smem = (size_t)(w.R * w.R + w.R) * sizeof(double);
  k_gram_inverse<<<1, 256, smem, s>>>(g, w.nmodes, mode, w.R, w.vinv64.get());
  ADATM_LAUNCH();
}

void update_factor(const double *M, uint64_t rows, float *A, __nv_bfloat16 *Ab, double *G_mode,
                   bool inner, AlsWork &w, cudaStream_t s) {
  UpdArgs u;
  u.split = 1;
  u.Md = M;
  u.M = nullptr;
  u.vinv = w.vinv64.get();
  u.A = A;
  u.rows = rows;
  u.R = w.R;
  u.ldr = w.ldr;
  u.part_gram = w.part_gram.get();
  u.part_max = w.part_max.get();
  const int nb = update_blocks(rows, w.R, w.nblocks);
  run_update(u, nb, s);
  k_finalize<<<finalize_blocks(w.R), 256, 0, s>>>(w.part_gram.get(), w.part_max.get(), nb, w.R, G_mode,
                               w.lambda.get(), w.iter.get());
  ADATM_LAUNCH();
  double *pi = inner ? w.part_inner.get() : nullptr;
  switch (lanes_for(w.R)) {
    case 4: k_scale<4><<<w.nblocks, 256, 0, s>>>(A, Ab, M, rows, w.R, w.ldr, w.lambda.get(), pi); break;
    case 8: k_scale<8><<<w.nblocks, 256, 0, s>>>(A, Ab, M, rows, w.R, w.ldr, w.lambda.get(), pi); break;
    case 16: k_scale<16><<<w.nblocks, 256, 0, s>>>(A, Ab, M, rows, w.R, w.ldr, w.lambda.get(), pi); break;
    default: k_scale<32><<<w.nblocks, 256, 0, s>>>(A, Ab, M, rows, w.R, w.ldr, w.lambda.get(), pi); break;
  }
  ADATM_LAUNCH();
  // BF16 factors were rounded after the Gram was taken: take it again from
  // the rounded rows, so the next modes' normal equations use the factor the
  // MTTKRPs read
  if (Ab) gram(A, rows, w.R, w.ldr, G_mode, w, s, true);
}

void fit(const GramSet &g, AlsWork &w, cudaStream_t s) {
  k_fit<<<1, 256, 0, s>>>(g, w.nmodes, w.R, w.lambda.get(), w.part_inner.get(), w.nblocks,
                          w.scalars.get(), w.fit_trace.get(), w.max_trace, w.iter.get());
  ADATM_LAUNCH();
}

// ---------------------------------------------------------------------------
// G = A^T A without any device allocation.
//
// For callers that cannot allocate device memory at the point of the call:
// a host whose caching allocator already holds nearly all of HBM (cudaMalloc
// would fail there), or a loop that must not pay cudaFree's implicit
// device-wide synchronisation. The per-block partial Grams and column maxima
// live in a fixed file-scope device array instead of an AlsWork, which bounds
// the rank to kNoallocMaxR columns and the row blocks to kNoallocBlocks.
//
// Every block of k_update writes its whole partial before k_finalize reads
// it, so nothing in the scratch has to start at zero. The scratch is shared
// by all calls on one device: calls that overlap in time (two host threads,
// or streams not ordered against each other) race on it. The first call on a
// device resolves the scratch address (and sets kernel attributes), which is
// set-up work a caller should do once before any stream capture.
// ---------------------------------------------------------------------------
constexpr int kNoallocMaxR = 64;
constexpr int kNoallocBlocks = 64;
constexpr size_t kNoallocGramDoubles = (size_t)kNoallocBlocks * kNoallocMaxR * kNoallocMaxR;
constexpr size_t kNoallocDoubles = kNoallocGramDoubles + (size_t)kNoallocBlocks * kNoallocMaxR;
constexpr int kNoallocMaxDevices = 64;

// 2 MiB of partial Grams + 32 KiB of column maxima.
static __device__ __align__(256) double g_noalloc_scratch[kNoallocDoubles];

namespace {

struct NoallocSlot {
  std::mutex mu;
  bool ready = false;
  double *ptr = nullptr;
};
NoallocSlot g_noalloc_slots[kNoallocMaxDevices];

// Device address of the scratch on the current device, resolved on the
// first successful call and kept; a failed set-up is not kept, so a later
// call tries again. cudaDeviceReset unloads the module that holds the
// scratch: the kept address is then stale, so a process must not call the
// entry point again after resetting the device.
double *noalloc_scratch() {
  int dev = 0;
  ADATM_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoallocMaxDevices) throw BadInput("device ordinal above the scratch table");
  NoallocSlot &slot = g_noalloc_slots[dev];
  std::lock_guard<std::mutex> lk(slot.mu);
  if (!slot.ready) {
    void *p = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (err != cudaSuccess) {
      cudaGetLastError();
      throw CudaError(std::string("scratch set-up failed: ") + cudaGetErrorString(err));
    }
    set_attributes();
    slot.ptr = static_cast<double *>(p);
    slot.ready = true;
  }
  return slot.ptr;
}

}  // namespace

int gram_noalloc_max_rank() { return kNoallocMaxR; }

void gram_noalloc(const float *A, uint64_t rows, int R, int ldr, double *G, cudaStream_t s) {
  if (R < 1 || R > kNoallocMaxR)
    throw BadInput("adatm_gram_noalloc: R = " + std::to_string(R) + " is outside 1.." +
                   std::to_string(kNoallocMaxR) + ", the columns its fixed scratch holds");
  if (ldr < R || ldr % 4 != 0) throw BadInput("adatm_gram_noalloc: ldr must be >= R and a multiple of 4");
  if (((uintptr_t)A & 15) != 0) throw BadInput("adatm_gram_noalloc: A must be 16-byte aligned");
  double *scratch = noalloc_scratch();
  UpdArgs u;
  u.split = 1;
  u.Md = nullptr;
  u.M = A;
  u.vinv = nullptr;
  u.A = nullptr;
  u.rows = rows;
  u.R = R;
  u.ldr = ldr;
  u.part_gram = scratch;
  u.part_max = scratch + kNoallocGramDoubles;
  const int nb = update_blocks(rows, R, kNoallocBlocks);
  run_update(u, nb, s);
  k_finalize<<<finalize_blocks(R), 256, 0, s>>>(u.part_gram, u.part_max, nb, R, G, nullptr,
                                                nullptr);
  ADATM_LAUNCH();
}

}  // namespace adatm
