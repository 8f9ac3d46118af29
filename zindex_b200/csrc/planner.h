// Learned launch planner: a two-layer FP32 perceptron trained on the GPU.
//
// The network maps a feature vector x (index geometry, batch shape and one
// candidate launch configuration) to a predicted cost y (log of the time per
// seed). Parameters, in this order: W1 (hidden x inputs, row-major), b1
// (hidden), w2 (hidden), b2 (1); h = relu(W1 x + b1), y = w2 . h + b2.
// Loss over n samples: L = (1 / 2n) sum (y_i - t_i)^2.
//
// Forward, backward and the Adam update are hand-written kernels
// (planner.cu). Gradients are reduced in a fixed order (per-block sums, then a
// sum over blocks in block order), so they are deterministic and comparable
// with a CPU computation to FP32 rounding. The planner only chooses launch
// configurations; it never touches the filter arithmetic.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

namespace zx {

class Mlp {
 public:
  Mlp(int device, int inputs, int hidden, uint64_t seed);
  ~Mlp();
  Mlp(const Mlp&) = delete;
  Mlp& operator=(const Mlp&) = delete;

  int inputs() const { return d_; }
  int hidden() const { return h_; }
  uint64_t param_count() const { return (uint64_t)h_ * d_ + 2ull * h_ + 1; }
  std::vector<float> params();
  void set_params(const float* p, uint64_t count);
  // Loss and its gradient (host arrays: x n x inputs row-major, t n).
  float loss_grad(const float* x, const float* t, uint64_t n, float* grad);
  // Full-batch Adam for `epochs` steps; returns the final loss.
  float train(const float* x, const float* t, uint64_t n, int epochs, float lr);
  void predict(const float* x, uint64_t n, float* y);

 private:
  void upload(const float* x, const float* t, uint64_t n);
  float step_grad(uint64_t n);  // grads of the resident batch into d_grad_, returns loss

  int device_, d_, h_;
  cudaStream_t stream_ = nullptr;
  float *d_params_ = nullptr, *d_grad_ = nullptr, *d_m_ = nullptr, *d_v_ = nullptr;
  float *d_x_ = nullptr, *d_t_ = nullptr, *d_y_ = nullptr, *d_partial_ = nullptr;
  float* d_loss_ = nullptr;
  uint64_t cap_n_ = 0;
  uint64_t adam_t_ = 0;
};

}  // namespace zx
