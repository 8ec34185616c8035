// mlp.hpp -- the learned plan model's network (see mlp.cu).
#pragma once

#include <vector>

#include "common.cuh"

namespace adatm {

class Mlp {
 public:
  // widths: input, hidden..., 1. Weights He-uniform from `seed`.
  Mlp(const std::vector<int> &widths, uint64_t seed, cudaStream_t s);
  uint64_t nparams() const { return nparams_; }
  const std::vector<int> &widths() const { return widths_; }
  void set_params(const float *host);  // also resets the optimizer state
  void get_params(float *host) const;
  // Y[B] = net(X[B x in]) (host buffers).
  void forward(const float *X, int B, float *Y);
  // Mean squared error of net(X) against T and its gradient (host, nparams
  // floats, same layout as the parameters; may be null).
  double gradient(const float *X, const float *T, int B, float *grad);
  // Adam on minibatches of `batch` rows drawn in a seeded order; returns the
  // mean loss of the last epoch.
  double train(const float *X, const float *T, uint64_t n, int epochs, int batch, float lr,
               uint64_t seed);

 private:
  void reserve(int B);
  void forward_dev(int B);
  double backward_dev(int B);

  std::vector<int> widths_;
  cudaStream_t s_;
  std::vector<uint64_t> woff_, boff_;
  uint64_t nparams_ = 0;
  uint64_t step_ = 0;
  int cap_ = 0;
  DevBuf<float> params_, grads_, m_, v_, target_, sq_;
  std::vector<DevBuf<float>> acts_, pre_, dacts_;
};

}  // namespace adatm
