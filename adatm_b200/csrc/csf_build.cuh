// csf_build.cuh -- device COO tensors and CSF construction on the GPU.
#pragma once

#include <vector>

#include "common.cuh"

namespace adatm {

// A COO tensor resident in HBM: per-mode uint32 index arrays and FP64 values.
struct DevCoo {
  int nmodes = 0;
  uint64_t nnz = 0;
  uint64_t dims[kMaxModes] = {0};
  DevBuf<uint32_t> idx[kMaxModes];
  DevBuf<double> vals;
};

// A CSF tree resident in HBM (one tile, no tiling: SPLATT_NOTILE).
struct DevCsf {
  int nmodes = 0;
  uint64_t nnz = 0;
  uint64_t dims[kMaxModes] = {0};      // per mode (not permuted)
  uint64_t dim_perm[kMaxModes] = {0};  // dim_perm[l] = mode stored at level l
  uint64_t nfibs[kMaxModes] = {0};
  DevBuf<uint32_t> fptr[kMaxModes];    // levels 0..N-2, nfibs[l]+1 entries
  DevBuf<uint32_t> fids[kMaxModes];    // levels 0..N-1 (0 = root ids)
  DevBuf<double> vals64;               // leaf values, FP64 (bit-exact copy)
  DevBuf<float> vals32;                // leaf values, FP32 (compute copy)
  // Close depth of every node of levels 1..N-1: how many ancestor levels end
  // together with it (0 = not the last child of its parent; 1 = last child,
  // its parent not the last child of its own parent; ...). A walk that reads
  // it knows where every node of every level above closes without touching
  // fptr.
  DevBuf<uint8_t> cdepth[kMaxModes];
  size_t device_bytes() const;
};

// Bit layout of a lexicographic sort key: levels packed leaf-first into up
// to three 64-bit words, no level straddling two words.
struct KeySpec {
  int nlev = 0;
  int words = 1;
  int word[kMaxModes] = {0};
  int shift[kMaxModes] = {0};
  int bits[kMaxModes] = {0};
  uint64_t prefix_mask[kMaxModes][3] = {{0}};  // bits of levels 0..l per word
  int used_bits[3] = {0, 0, 0};
};
KeySpec make_key_spec(int nmodes, const uint64_t *dims, const uint64_t *perm);

// Upload a host COO (64-bit indices, mode-major pointers) and narrow it to
// uint32. Throws BadInput for indices out of range.
void coo_upload(DevCoo &out, int nmodes, uint64_t nnz, const uint64_t *dims,
                const uint64_t *const *inds, const double *vals, cudaStream_t s);

// Sum duplicates in input order and compact empty slices of every mode,
// producing a new COO whose nonzeros are in natural (mode 0..N-1) order.
void coo_clean(const DevCoo &in, DevCoo &out, cudaStream_t s);

// Seeded synthetic tensor: indices per mode uniform (alpha <= 0) or bounded
// Zipf(alpha) with P(k) proportional to (k+1)^-alpha, values uniform(0,1)
// (value_kind 0) or lognormal(mu, sigma) (value_kind 1). Duplicates are NOT
// summed here; run coo_clean afterwards.
void coo_generate(DevCoo &out, int nmodes, const uint64_t *dims, uint64_t nnz,
                  const double *alpha, int value_kind, double mu, double sigma,
                  uint64_t seed, cudaStream_t s);

// Build the CSF of `coo` in level order `perm` (bit-exact with the
// reference's p_csf_alloc_untiled on a cleaned COO).
void csf_build(const DevCoo &coo, const uint64_t *perm, DevCsf &out, cudaStream_t s);

// Fiber counts per level of the tree in order `perm` (count_nfibs), without
// building the arrays. nfibs[N-1] = nnz.
void csf_count(const DevCoo &coo, const uint64_t *perm, uint64_t *nfibs, cudaStream_t s);

// Copy a device CSF into host arrays in the reference layout (64-bit).
struct HostCsfArrays {
  std::vector<std::vector<uint64_t>> fptr, fids;
  std::vector<double> vals;
};
void csf_download(const DevCsf &c, HostCsfArrays &h, cudaStream_t s);

}  // namespace adatm
