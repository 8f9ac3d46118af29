// Two-layer FP32 perceptron of the launch planner: forward, backward and
// Adam kernels (see planner.h).
#include "planner.h"

#include <algorithm>
#include <cmath>

#include "engine.h"
#include "host/error.h"
#include "zx_hash.h"

namespace zx {

namespace {

constexpr int kMlpBlock = 64;  // samples per block
constexpr int kMaxInputs = 32, kMaxHidden = 64;  // shared memory of a block stays below 48 KB

// Forward and per-sample backward of one block of samples, then the block's
// gradient sums in sample order: partial[block][p] for every parameter p,
// partial_loss[block].
__global__ void mlp_grad_kernel(const float* __restrict__ prm, const float* __restrict__ x,
                                const float* __restrict__ t, uint64_t n, int D, int H,
                                float* __restrict__ partial, float* __restrict__ partial_loss) {
  extern __shared__ float sm[];
  float* xs = sm;                     // kMlpBlock x D
  float* hs = xs + kMlpBlock * D;     // kMlpBlock x H
  float* dz = hs + kMlpBlock * H;     // kMlpBlock x H
  float* dy = dz + kMlpBlock * H;     // kMlpBlock
  float* ls = dy + kMlpBlock;         // kMlpBlock
  const float* W1 = prm;
  const float* b1 = W1 + H * D;
  const float* w2 = b1 + H;
  const float b2 = w2[H];
  const int i = threadIdx.x;
  const uint64_t s = blockIdx.x * (uint64_t)kMlpBlock + i;
  const bool live = s < n;
  for (int k = 0; k < D; ++k) xs[i * D + k] = live ? x[s * D + k] : 0.f;
  float y = b2;
  for (int j = 0; j < H; ++j) {
    float z = b1[j];
    for (int k = 0; k < D; ++k) z = fmaf(W1[j * D + k], xs[i * D + k], z);
    const float h = z > 0.f ? z : 0.f;
    hs[i * H + j] = h;
    dz[i * H + j] = z > 0.f ? w2[j] : 0.f;
    y = fmaf(w2[j], h, y);
  }
  const float r = live ? y - t[s] : 0.f;
  const float g = r / (float)n;
  dy[i] = g;
  ls[i] = 0.5f * r * r / (float)n;
  for (int j = 0; j < H; ++j) dz[i * H + j] *= g;
  __syncthreads();
  const int P = H * D + 2 * H + 1;
  float* out = partial + (uint64_t)blockIdx.x * P;
  for (int p = i; p < P; p += kMlpBlock) {
    float acc = 0.f;
    if (p < H * D) {
      const int j = p / D, k = p % D;
      for (int q = 0; q < kMlpBlock; ++q) acc = fmaf(dz[q * H + j], xs[q * D + k], acc);
    } else if (p < H * D + H) {
      const int j = p - H * D;
      for (int q = 0; q < kMlpBlock; ++q) acc += dz[q * H + j];
    } else if (p < H * D + 2 * H) {
      const int j = p - H * D - H;
      for (int q = 0; q < kMlpBlock; ++q) acc = fmaf(dy[q], hs[q * H + j], acc);
    } else {
      for (int q = 0; q < kMlpBlock; ++q) acc += dy[q];
    }
    out[p] = acc;
  }
  if (i == 0) {
    float acc = 0.f;
    for (int q = 0; q < kMlpBlock; ++q) acc += ls[q];
    partial_loss[blockIdx.x] = acc;
  }
}

// grad[p] = sum over blocks, in block order, of partial[block][p]; thread 0
// also sums the losses.
__global__ void mlp_reduce_kernel(const float* __restrict__ partial,
                                  const float* __restrict__ partial_loss, uint32_t blocks, int P,
                                  float* __restrict__ grad, float* __restrict__ loss) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
    float acc = 0.f;
    for (uint32_t b = 0; b < blocks; ++b) acc += partial[(uint64_t)b * P + p];
    grad[p] = acc;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    float acc = 0.f;
    for (uint32_t b = 0; b < blocks; ++b) acc += partial_loss[b];
    *loss = acc;
  }
}

// Adam (Kingma and Ba, 2015) with bias correction.
__global__ void mlp_adam_kernel(float* __restrict__ prm, const float* __restrict__ grad,
                                float* __restrict__ m, float* __restrict__ v, int P, float lr,
                                float c1, float c2) {
  const float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
    const float g = grad[p];
    const float mm = beta1 * m[p] + (1.f - beta1) * g;
    const float vv = beta2 * v[p] + (1.f - beta2) * g * g;
    m[p] = mm;
    v[p] = vv;
    prm[p] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
  }
}

__global__ void mlp_forward_kernel(const float* __restrict__ prm, const float* __restrict__ x,
                                   uint64_t n, int D, int H, float* __restrict__ y) {
  const float* W1 = prm;
  const float* b1 = W1 + H * D;
  const float* w2 = b1 + H;
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < n;
       s += (uint64_t)gridDim.x * blockDim.x) {
    float out = w2[H];
    for (int j = 0; j < H; ++j) {
      float z = b1[j];
      for (int k = 0; k < D; ++k) z = fmaf(W1[j * D + k], x[s * D + k], z);
      out = fmaf(w2[j], z > 0.f ? z : 0.f, out);
    }
    y[s] = out;
  }
}

template <class T>
T* dalloc(uint64_t count) {
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, std::max<uint64_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    raise(kENoMem, std::string("planner: device allocation failed: ") + cudaGetErrorString(e));
  }
  return static_cast<T*>(p);
}

}  // namespace

Mlp::Mlp(int device, int inputs, int hidden, uint64_t seed)
    : device_(device), d_(inputs), h_(hidden) {
  check(inputs >= 1 && inputs <= kMaxInputs && hidden >= 1 && hidden <= kMaxHidden, kEInval,
        "planner network: 1..32 inputs and 1..64 hidden units");
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  const uint64_t P = param_count();
  d_params_ = dalloc<float>(P);
  d_grad_ = dalloc<float>(P);
  d_m_ = dalloc<float>(P);
  d_v_ = dalloc<float>(P);
  d_loss_ = dalloc<float>(1);
  // Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights from splitmix64, zero biases.
  std::vector<float> p(P, 0.f);
  uint64_t state = seed;
  auto uniform = [&](float a) {
    state += 0x9E3779B97F4A7C15ull;
    const uint64_t r = splitmix64(state);
    return (float)((double)(r >> 11) / 9007199254740992.0 * 2.0 - 1.0) * a;
  };
  for (int q = 0; q < h_ * d_; ++q) p[q] = uniform(1.f / std::sqrt((float)d_));
  for (int j = 0; j < h_; ++j) p[(uint64_t)h_ * d_ + h_ + j] = uniform(1.f / std::sqrt((float)h_));
  set_params(p.data(), P);
}

Mlp::~Mlp() {
  cudaSetDevice(device_);
  for (float* q : {d_params_, d_grad_, d_m_, d_v_, d_x_, d_t_, d_y_, d_partial_, d_loss_})
    if (q) cudaFree(q);
  if (stream_) cudaStreamDestroy(stream_);
}

std::vector<float> Mlp::params() {
  std::vector<float> p(param_count());
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  cuda_check(cudaMemcpyAsync(p.data(), d_params_, p.size() * 4, cudaMemcpyDeviceToHost, stream_),
             "D2H");
  cuda_check(cudaStreamSynchronize(stream_), "planner");
  return p;
}

void Mlp::set_params(const float* p, uint64_t count) {
  check(count == param_count(), kEInval, "planner parameter count mismatch");
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  cuda_check(cudaMemcpyAsync(d_params_, p, count * 4, cudaMemcpyHostToDevice, stream_), "H2D");
  cuda_check(cudaMemsetAsync(d_m_, 0, count * 4, stream_), "memset");
  cuda_check(cudaMemsetAsync(d_v_, 0, count * 4, stream_), "memset");
  cuda_check(cudaStreamSynchronize(stream_), "planner");
  adam_t_ = 0;
}

void Mlp::upload(const float* x, const float* t, uint64_t n) {
  check(n > 0, kEInval, "planner: no samples");
  if (n > cap_n_) {
    for (float* q : {d_x_, d_t_, d_y_, d_partial_})
      if (q) cudaFree(q);
    const uint64_t cap = std::max<uint64_t>(n, 256);
    d_x_ = dalloc<float>(cap * d_);
    d_t_ = dalloc<float>(cap);
    d_y_ = dalloc<float>(cap);
    const uint64_t blocks = (cap + kMlpBlock - 1) / kMlpBlock;
    d_partial_ = dalloc<float>(blocks * (param_count() + 1));
    cap_n_ = cap;
  }
  cuda_check(cudaMemcpyAsync(d_x_, x, n * d_ * 4, cudaMemcpyHostToDevice, stream_), "H2D");
  if (t) cuda_check(cudaMemcpyAsync(d_t_, t, n * 4, cudaMemcpyHostToDevice, stream_), "H2D");
}

float Mlp::step_grad(uint64_t n) {
  const uint32_t blocks = (uint32_t)((n + kMlpBlock - 1) / kMlpBlock);
  const int P = (int)param_count();
  const size_t smem = (size_t)kMlpBlock * (d_ + 2 * h_ + 2) * sizeof(float);
  float* partial_loss = d_partial_ + (uint64_t)blocks * P;
  mlp_grad_kernel<<<blocks, kMlpBlock, smem, stream_>>>(d_params_, d_x_, d_t_, n, d_, h_,
                                                        d_partial_, partial_loss);
  cuda_check(cudaGetLastError(), "mlp_grad_kernel");
  mlp_reduce_kernel<<<(P + 255) / 256, 256, 0, stream_>>>(d_partial_, partial_loss, blocks, P,
                                                          d_grad_, d_loss_);
  cuda_check(cudaGetLastError(), "mlp_reduce_kernel");
  return 0.f;
}

float Mlp::loss_grad(const float* x, const float* t, uint64_t n, float* grad) {
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  upload(x, t, n);
  step_grad(n);
  float loss = 0.f;
  if (grad)
    cuda_check(cudaMemcpyAsync(grad, d_grad_, param_count() * 4, cudaMemcpyDeviceToHost, stream_),
               "D2H");
  cuda_check(cudaMemcpyAsync(&loss, d_loss_, 4, cudaMemcpyDeviceToHost, stream_), "D2H");
  cuda_check(cudaStreamSynchronize(stream_), "planner");
  return loss;
}

float Mlp::train(const float* x, const float* t, uint64_t n, int epochs, float lr) {
  check(epochs >= 0 && lr > 0.f, kEInval, "planner: epochs >= 0 and a positive learning rate");
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  upload(x, t, n);
  const int P = (int)param_count();
  for (int e = 0; e < epochs; ++e) {
    step_grad(n);
    ++adam_t_;
    const float c1 = 1.f - std::pow(0.9f, (float)adam_t_);
    const float c2 = 1.f - std::pow(0.999f, (float)adam_t_);
    mlp_adam_kernel<<<(P + 255) / 256, 256, 0, stream_>>>(d_params_, d_grad_, d_m_, d_v_, P, lr,
                                                          c1, c2);
    cuda_check(cudaGetLastError(), "mlp_adam_kernel");
  }
  step_grad(n);
  float loss = 0.f;
  cuda_check(cudaMemcpyAsync(&loss, d_loss_, 4, cudaMemcpyDeviceToHost, stream_), "D2H");
  cuda_check(cudaStreamSynchronize(stream_), "planner");
  return loss;
}

void Mlp::predict(const float* x, uint64_t n, float* y) {
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  upload(x, nullptr, n);
  const int grid = (int)std::min<uint64_t>((n + 127) / 128, 1024);
  mlp_forward_kernel<<<grid, 128, 0, stream_>>>(d_params_, d_x_, n, d_, h_, d_y_);
  cuda_check(cudaGetLastError(), "mlp_forward_kernel");
  cuda_check(cudaMemcpyAsync(y, d_y_, n * 4, cudaMemcpyDeviceToHost, stream_), "D2H");
  cuda_check(cudaStreamSynchronize(stream_), "planner");
}

}  // namespace zx
