// common.cuh -- shared definitions for the B200 AdaTM library.
//
// Device layout conventions used throughout:
//  * tensor indices are uint32 on the device (dims and nnz must stay below
//    2^32 - 1; the C-ABI rejects larger inputs with SPLATT_ERROR_BADINPUT);
//  * dense row matrices (factors, MTTKRP outputs, memo rows) are row-major
//    with a padded leading dimension ldr = round_up(R, 4) floats, so every
//    lane of a row group moves one 16-byte float4 (or 8-byte bf16x4);
//  * CSF levels follow the reference layout (include/splatt.h:235-287):
//    fptr[l] has nfibs[l]+1 entries and points into level l+1 (into the
//    nonzeros for l = N-2); fids[l] holds the index of every node, with
//    fids[0] kept explicitly (root ids) on the device.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <stdexcept>
#include <string>

namespace adatm {

constexpr int kMaxModes = 8;  // device kernels support orders 3..8

struct CudaError : std::runtime_error {
  explicit CudaError(const std::string &s) : std::runtime_error(s) {}
};
struct BadInput : std::runtime_error {
  explicit BadInput(const std::string &s) : std::runtime_error(s) {}
};
struct NoMemory : std::runtime_error {
  explicit NoMemory(const std::string &s) : std::runtime_error(s) {}
};

inline void check_cuda(cudaError_t e, const char *what, const char *file, int line) {
  if (e == cudaSuccess) return;
  char buf[512];
  snprintf(buf, sizeof(buf), "%s failed at %s:%d: %s", what, file, line, cudaGetErrorString(e));
  if (e == cudaErrorMemoryAllocation) throw NoMemory(buf);
  throw CudaError(buf);
}

#define ADATM_CUDA(call) ::adatm::check_cuda((call), #call, __FILE__, __LINE__)
#define ADATM_LAUNCH() ::adatm::check_cuda(cudaGetLastError(), "kernel launch", __FILE__, __LINE__)

inline int ldr_of(uint64_t R) { return (int)((R + 3) / 4 * 4); }

// (not volatile: a pure function of the lane, so the compiler may reuse it)
__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Exclusive device-wide prefix sum of n uint32 values (scan.cu). `tmp` must
// hold scan_tmp_words(n) uint32 of scratch. Values are summed in uint32.
size_t scan_tmp_words(size_t n);
void exclusive_scan_u32(const uint32_t *in, uint32_t *out, size_t n, uint32_t *tmp,
                        cudaStream_t stream);

// Simple RAII device buffer.
template <typename T>
struct DevBuf {
  T *p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  explicit DevBuf(size_t count) { alloc(count); }
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  DevBuf(DevBuf &&o) noexcept : p(o.p), n(o.n) {
    o.p = nullptr;
    o.n = 0;
  }
  DevBuf &operator=(DevBuf &&o) noexcept {
    if (this != &o) {
      reset();
      p = o.p;
      n = o.n;
      o.p = nullptr;
      o.n = 0;
    }
    return *this;
  }
  ~DevBuf() { reset(); }
  void alloc(size_t count) {
    reset();
    n = count;
    if (count) ADATM_CUDA(cudaMalloc(&p, count * sizeof(T)));
  }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  T *get() const { return p; }
  size_t bytes() const { return n * sizeof(T); }
};

}  // namespace adatm
