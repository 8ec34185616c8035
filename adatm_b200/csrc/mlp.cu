// mlp.cu -- the learned plan model: a small fully connected network (ReLU
// hidden layers, one linear output) that maps a candidate plan's features to
// its predicted log sweep time. Inference, gradients and Adam training run
// on the GPU with the kernels below; the analytic cost model of the
// reference (adatm_bench.c:145-272) stays the fallback.
//
// Parameters live in one FP32 device buffer, layer by layer: W_l (out x in,
// row-major) then b_l (out). The sizes are tiny (tens of units, batches of a
// few thousand rows), so every kernel maps one thread to one output element.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "mlp.hpp"

namespace adatm {

namespace {

constexpr int kThreads = 256;

unsigned blocks_for(uint64_t n) { return (unsigned)std::max<uint64_t>(1, (n + kThreads - 1) / kThreads); }

// Z[i, j] = sum_k A[i, k] W[j, k] + b[j]; H = relu(Z) when relu != 0.
__global__ void k_linear(const float *A, const float *W, const float *b, int B, int in, int out,
                         int relu, float *Z, float *H) {
  const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (uint64_t)B * out) return;
  const int i = (int)(e / out), j = (int)(e % out);
  const float *a = A + (size_t)i * in;
  const float *w = W + (size_t)j * in;
  float s = b[j];
  for (int k = 0; k < in; ++k) s = fmaf(a[k], w[k], s);
  Z[e] = s;
  H[e] = relu ? fmaxf(s, 0.f) : s;
}

// dY = 2 (Y - T) / B; per-row squared error for the loss.
__global__ void k_mse_grad(const float *Y, const float *T, int B, float *dY, float *sq) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B) return;
  const float r = Y[i] - T[i];
  dY[i] = 2.f * r / (float)B;
  sq[i] = r * r;
}

// dZ = dH * relu'(Z) (in place on dH when relu).
__global__ void k_relu_back(const float *Z, float *dH, uint64_t n) {
  const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n && Z[e] <= 0.f) dH[e] = 0.f;
}

// dW[j, k] = sum_i dZ[i, j] A[i, k]; db[j] = sum_i dZ[i, j].
__global__ void k_weight_grad(const float *dZ, const float *A, int B, int in, int out, float *dW,
                              float *db) {
  const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t nw = (uint64_t)out * in;
  if (e < nw) {
    const int j = (int)(e / in), k = (int)(e % in);
    float s = 0.f;
    for (int i = 0; i < B; ++i) s = fmaf(dZ[(size_t)i * out + j], A[(size_t)i * in + k], s);
    dW[e] = s;
  } else if (e < nw + out) {
    const int j = (int)(e - nw);
    float s = 0.f;
    for (int i = 0; i < B; ++i) s += dZ[(size_t)i * out + j];
    db[j] = s;
  }
}

// dA[i, k] = sum_j dZ[i, j] W[j, k].
__global__ void k_input_grad(const float *dZ, const float *W, int B, int in, int out, float *dA) {
  const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (uint64_t)B * in) return;
  const int i = (int)(e / in), k = (int)(e % in);
  float s = 0.f;
  for (int j = 0; j < out; ++j) s = fmaf(dZ[(size_t)i * out + j], W[(size_t)j * in + k], s);
  dA[e] = s;
}

// Adam (Kingma & Ba 2015) with bias correction.
__global__ void k_adam(float *p, const float *g, float *m, float *v, uint64_t n, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
  const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const float gi = g[e];
  const float mi = b1 * m[e] + (1.f - b1) * gi;
  const float vi = b2 * v[e] + (1.f - b2) * gi * gi;
  m[e] = mi;
  v[e] = vi;
  p[e] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// Rows idx[0..B) of X (n x in) and T into contiguous batch buffers.
__global__ void k_gather_rows(const float *X, const float *T, const uint32_t *idx, int B, int in,
                              float *Xb, float *Tb) {
  const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (uint64_t)B * in) return;
  const int i = (int)(e / in), k = (int)(e % in);
  Xb[e] = X[(size_t)idx[i] * in + k];
  if (k == 0) Tb[i] = T[idx[i]];
}

uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace

Mlp::Mlp(const std::vector<int> &widths, uint64_t seed, cudaStream_t s) : widths_(widths), s_(s) {
  if (widths.size() < 2) throw BadInput("the network needs an input and an output width");
  if (widths.back() != 1) throw BadInput("the network predicts one value per row");
  for (int w : widths)
    if (w < 1 || w > 4096) throw BadInput("layer width out of range");
  uint64_t off = 0;
  for (size_t l = 0; l + 1 < widths.size(); ++l) {
    woff_.push_back(off);
    off += (uint64_t)widths[l + 1] * widths[l];
    boff_.push_back(off);
    off += (uint64_t)widths[l + 1];
  }
  nparams_ = off;
  params_.alloc(nparams_);
  grads_.alloc(nparams_);
  m_.alloc(nparams_);
  v_.alloc(nparams_);
  // He-uniform weights from the seeded generator, zero biases
  std::vector<float> h(nparams_, 0.f);
  for (size_t l = 0; l + 1 < widths.size(); ++l) {
    const double bound = std::sqrt(6.0 / widths[l]);
    const uint64_t n = (uint64_t)widths[l + 1] * widths[l];
    for (uint64_t i = 0; i < n; ++i) {
      const double u = (double)(mix64(seed * 0x100000001B3ull + woff_[l] + i) >> 11) * 0x1.0p-53;
      h[woff_[l] + i] = (float)((2.0 * u - 1.0) * bound);
    }
  }
  set_params(h.data());
}

void Mlp::set_params(const float *host) {
  ADATM_CUDA(cudaMemcpyAsync(params_.get(), host, nparams_ * sizeof(float), cudaMemcpyHostToDevice, s_));
  ADATM_CUDA(cudaMemsetAsync(m_.get(), 0, nparams_ * sizeof(float), s_));
  ADATM_CUDA(cudaMemsetAsync(v_.get(), 0, nparams_ * sizeof(float), s_));
  step_ = 0;
  ADATM_CUDA(cudaStreamSynchronize(s_));
}

void Mlp::get_params(float *host) const {
  ADATM_CUDA(cudaMemcpyAsync(host, params_.get(), nparams_ * sizeof(float), cudaMemcpyDeviceToHost, s_));
  ADATM_CUDA(cudaStreamSynchronize(s_));
}

void Mlp::reserve(int B) {
  if (B <= cap_) return;
  cap_ = B;
  const size_t L = widths_.size();
  acts_.clear();
  pre_.clear();
  dacts_.clear();
  acts_.resize(L);
  pre_.resize(L);
  dacts_.resize(L);
  for (size_t l = 0; l < L; ++l) {
    acts_[l].alloc((size_t)B * widths_[l]);
    pre_[l].alloc((size_t)B * widths_[l]);
    dacts_[l].alloc((size_t)B * widths_[l]);
  }
  target_.alloc(B);
  sq_.alloc(B);
}

void Mlp::forward_dev(int B) {
  const size_t L = widths_.size();
  for (size_t l = 0; l + 1 < L; ++l) {
    const int in = widths_[l], out = widths_[l + 1];
    const int relu = (l + 2 < L) ? 1 : 0;
    k_linear<<<blocks_for((uint64_t)B * out), kThreads, 0, s_>>>(
        acts_[l].get(), params_.get() + woff_[l], params_.get() + boff_[l], B, in, out, relu,
        pre_[l + 1].get(), acts_[l + 1].get());
    ADATM_LAUNCH();
  }
}

double Mlp::backward_dev(int B) {
  const size_t L = widths_.size();
  k_mse_grad<<<blocks_for(B), kThreads, 0, s_>>>(acts_[L - 1].get(), target_.get(), B,
                                                  dacts_[L - 1].get(), sq_.get());
  ADATM_LAUNCH();
  for (size_t l = L - 1; l >= 1; --l) {
    const int in = widths_[l - 1], out = widths_[l];
    if (l + 1 < L) {  // hidden layer: through the ReLU
      k_relu_back<<<blocks_for((uint64_t)B * out), kThreads, 0, s_>>>(pre_[l].get(), dacts_[l].get(),
                                                                     (uint64_t)B * out);
      ADATM_LAUNCH();
    }
    k_weight_grad<<<blocks_for((uint64_t)out * in + out), kThreads, 0, s_>>>(
        dacts_[l].get(), acts_[l - 1].get(), B, in, out, grads_.get() + woff_[l - 1],
        grads_.get() + boff_[l - 1]);
    ADATM_LAUNCH();
    if (l > 1) {
      k_input_grad<<<blocks_for((uint64_t)B * in), kThreads, 0, s_>>>(
          dacts_[l].get(), params_.get() + woff_[l - 1], B, in, out, dacts_[l - 1].get());
      ADATM_LAUNCH();
    }
  }
  std::vector<float> sq(B);
  ADATM_CUDA(cudaMemcpyAsync(sq.data(), sq_.get(), B * sizeof(float), cudaMemcpyDeviceToHost, s_));
  ADATM_CUDA(cudaStreamSynchronize(s_));
  double loss = 0;
  for (float x : sq) loss += x;
  return loss / B;
}

void Mlp::forward(const float *X, int B, float *Y) {
  if (B <= 0) return;
  reserve(B);
  ADATM_CUDA(cudaMemcpyAsync(acts_[0].get(), X, (size_t)B * widths_[0] * sizeof(float),
                             cudaMemcpyHostToDevice, s_));
  forward_dev(B);
  ADATM_CUDA(cudaMemcpyAsync(Y, acts_.back().get(), (size_t)B * sizeof(float), cudaMemcpyDeviceToHost,
                             s_));
  ADATM_CUDA(cudaStreamSynchronize(s_));
}

double Mlp::gradient(const float *X, const float *T, int B, float *grad) {
  if (B <= 0) throw BadInput("empty batch");
  reserve(B);
  ADATM_CUDA(cudaMemcpyAsync(acts_[0].get(), X, (size_t)B * widths_[0] * sizeof(float),
                             cudaMemcpyHostToDevice, s_));
  ADATM_CUDA(cudaMemcpyAsync(target_.get(), T, (size_t)B * sizeof(float), cudaMemcpyHostToDevice, s_));
  forward_dev(B);
  const double loss = backward_dev(B);
  if (grad) {
    ADATM_CUDA(cudaMemcpyAsync(grad, grads_.get(), nparams_ * sizeof(float), cudaMemcpyDeviceToHost, s_));
    ADATM_CUDA(cudaStreamSynchronize(s_));
  }
  return loss;
}

double Mlp::train(const float *X, const float *T, uint64_t n, int epochs, int batch, float lr,
                  uint64_t seed) {
  if (n == 0 || batch <= 0 || epochs <= 0) throw BadInput("empty training set or schedule");
  const int in = widths_[0];
  const int B = (int)std::min<uint64_t>((uint64_t)batch, n);
  reserve(B);
  DevBuf<float> Xd((size_t)n * in), Td(n);
  DevBuf<uint32_t> idx_d(n);
  ADATM_CUDA(cudaMemcpyAsync(Xd.get(), X, (size_t)n * in * sizeof(float), cudaMemcpyHostToDevice, s_));
  ADATM_CUDA(cudaMemcpyAsync(Td.get(), T, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, s_));
  std::vector<uint32_t> order(n);
  for (uint64_t i = 0; i < n; ++i) order[i] = (uint32_t)i;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  double last = 0;
  for (int ep = 0; ep < epochs; ++ep) {
    for (uint64_t i = n - 1; i > 0; --i) {  // Fisher-Yates with the seeded generator
      const uint64_t j = mix64(seed * 0x9E3779B97F4A7C15ull + (uint64_t)ep * n + i) % (i + 1);
      std::swap(order[i], order[j]);
    }
    ADATM_CUDA(cudaMemcpyAsync(idx_d.get(), order.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice,
                               s_));
    double sum = 0;
    uint64_t rows = 0;
    for (uint64_t off = 0; off + B <= n; off += B) {
      k_gather_rows<<<blocks_for((uint64_t)B * in), kThreads, 0, s_>>>(
          Xd.get(), Td.get(), idx_d.get() + off, B, in, acts_[0].get(), target_.get());
      ADATM_LAUNCH();
      forward_dev(B);
      sum += backward_dev(B) * B;
      rows += B;
      ++step_;
      const float c1 = 1.f - std::pow(b1, (float)step_);
      const float c2 = 1.f - std::pow(b2, (float)step_);
      k_adam<<<blocks_for(nparams_), kThreads, 0, s_>>>(params_.get(), grads_.get(), m_.get(), v_.get(),
                                                        nparams_, lr, b1, b2, eps, c1, c2);
      ADATM_LAUNCH();
    }
    last = rows ? sum / rows : 0;
  }
  ADATM_CUDA(cudaStreamSynchronize(s_));
  return last;
}

}  // namespace adatm
