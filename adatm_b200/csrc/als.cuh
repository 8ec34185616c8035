// als.cuh -- the dense part of one CP-ALS mode update on the GPU
// (cpd_als_iterate_adaptive, adatm_cpd.c:320-335, and the fit,
// adatm_cpd.c:59-200). FP64 is kept for the R x R Gram Hadamard product, its
// Cholesky inverse, lambda and the fit; the I x R rows stay FP32.
#pragma once

#include "common.cuh"

namespace adatm {

struct AlsWork {
  int nmodes = 0, R = 0, ldr = 0;
  int nblocks = 0;                       // row blocks of the update kernels
  DevBuf<double> vinv64;                 // R x R
  DevBuf<double> part_gram;              // nblocks x R x R
  DevBuf<double> part_max;               // nblocks x R
  DevBuf<double> part_inner;             // nblocks x R
  DevBuf<double> lambda;                 // R
  DevBuf<double> scalars;                // [0] ttnormsq, [1] fit, [2] norm, [3] inner
  DevBuf<int> iter;                      // ALS iteration counter (device)
  DevBuf<double> fit_trace;              // per-iteration fits
  DevBuf<double> frob_part;              // partial sums of ||X||^2
  int max_trace = 0;
  void init(int nmodes_, int R_, int nblocks_, int max_iters);
};

struct GramSet {
  const double *G[kMaxModes];
};

// A (I x ldr, fp32) from the seeded generator: entry (i, r) of mode m is
// uniform [0,1) from mix64(mix64(seed * 0x100000001B3 + m) + i * R + r).
void factor_init_device(float *A, __nv_bfloat16 *Ab, uint64_t rows, int R, int ldr, uint64_t seed,
                        uint64_t mode, cudaStream_t s);
// G = A^T A (R x R, FP64 result): TF32 tensor-core tiles with FP32
// accumulation per row group, FP64 across groups; FP32 rows take three TF32
// products (big/remainder split), BF16-valued rows (bf16_rows) one exact one.
void gram(const float *A, uint64_t rows, int R, int ldr, double *G, AlsWork &w, cudaStream_t s,
          bool bf16_rows = false);
// sum of squares of the tensor values -> w.scalars[0]
void frob_sq(const double *vals, uint64_t n, AlsWork &w, cudaStream_t s);
// V = Hadamard of all G[n], n != mode; write V^-1 (fp64).
void gram_inverse(const GramSet &g, int mode, AlsWork &w, cudaStream_t s);
// A = normalize(M * V^-1) (M: the FP64 MTTKRP rows); updates lambda (2-norm on the first iteration,
// max-norm floored at 1 afterwards), G_mode and, when `inner` is set, the
// partial inner products <A, M> of the fit. A is fp32; with a bf16 copy (Ab
// non-null) the rows are rounded to bf16 in both copies and G_mode is taken
// from the rounded rows.
void update_factor(const double *M, uint64_t rows, float *A, __nv_bfloat16 *Ab, double *G_mode,
                   bool inner, AlsWork &w, cudaStream_t s);
// fit = 1 - sqrt(||X||^2 + ||Z||^2 - 2<X,Z>) / ||X||, stored in
// w.scalars[1] and w.fit_trace[iter]; advances w.iter.
void fit(const GramSet &g, AlsWork &w, cudaStream_t s);
// G = A^T A in FP64 like gram(), with its partial sums in a fixed device
// array instead of an AlsWork: no device allocation. R <= gram_noalloc_max_rank();
// calls that overlap in time on one device race on the shared array.
void gram_noalloc(const float *A, uint64_t rows, int R, int ldr, double *G, cudaStream_t s);
int gram_noalloc_max_rank();
// Round fp32 rows to bf16 (rows x ldr) into Ab and write the rounded values
// back to A: with BF16 factors the rounded value is the factor everywhere.
void to_bf16(float *A, __nv_bfloat16 *Ab, uint64_t rows, int ldr, cudaStream_t s);

}  // namespace adatm
