// Learned schedule cost model: a small FP32 MLP (in -> H -> H -> H -> 1,
// ReLU) trained and evaluated with hand-written CUDA kernels.
//
// It predicts log(kernel time) from DAG features plus a candidate schedule;
// the autotuner uses it to pick a schedule without timing every candidate.
// The network is small (hidden 256), so the kernels are plain SIMT FFMA:
//   * gemm: C[M,N] = op(A)[M,K] * op(B)[K,N] (+ bias, ReLU) with 64x64 output
//     tiles, 16-deep K tiles staged in shared memory, 4x4 outputs per thread;
//     op() = transpose flags, which give both backward products without
//     materializing transposes;
//   * relu_backward, mse (loss + gradient), column sums (bias gradients),
//     Adam (one fused update over the flat parameter vector).
// Parameters live in one flat device array: W1 b1 W2 b2 ... Wout bout, each
// W stored row-major [fan_in, fan_out].
#include "mlp.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "device.h"

namespace bsz {
namespace {

constexpr int TM = 64, TN = 64, TK = 16;

// C = op(A) * op(B) (+ bias[N]) (ReLU).  A is [M,K] (TA=0) or [K,M] (TA=1);
// B is [K,N] (TB=0) or [N,K] (TB=1).  All row-major.  accumulate: C += result.
template <int TA, int TB>
__global__ void __launch_bounds__(256)
k_gemm(const float* __restrict__ A, const float* __restrict__ B, float* __restrict__ C,
       const float* __restrict__ bias, int M, int N, int K, int relu, int accumulate) {
  __shared__ float As[TK][TM + 4];
  __shared__ float Bs[TK][TN + 4];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += TK) {
    for (int i = threadIdx.x; i < TK * TM; i += 256) {
      int kk = i / TM, mm = i % TM;
      int m = m0 + mm, k = k0 + kk;
      float v = 0.f;
      if (m < M && k < K) v = TA ? A[(size_t)k * M + m] : A[(size_t)m * K + k];
      As[kk][mm] = v;
    }
    for (int i = threadIdx.x; i < TK * TN; i += 256) {
      int kk = i / TN, nn = i % TN;
      int n = n0 + nn, k = k0 + kk;
      float v = 0.f;
      if (n < N && k < K) v = TB ? B[(size_t)n * K + k] : B[(size_t)k * N + n];
      Bs[kk][nn] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < TK; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int m = m0 + ty * 4 + i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int n = n0 + tx * 4 + j;
      if (n >= N) continue;
      float v = acc[i][j];
      if (bias) v += bias[n];
      if (relu) v = fmaxf(v, 0.f);
      float* c = C + (size_t)m * N + n;
      *c = accumulate ? *c + v : v;
    }
  }
}

// dZ = dH * (H > 0)
__global__ void k_relu_backward(float* __restrict__ d, const float* __restrict__ h, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && h[i] <= 0.f) d[i] = 0.f;
}

// loss = mean((p - t)^2), dp = 2 (p - t) / n
__global__ void k_mse(const float* __restrict__ p, const float* __restrict__ t, float* __restrict__ dp,
                      float* __restrict__ loss, int n) {
  __shared__ float part[256];
  float s = 0.f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    float e = p[i] - t[i];
    s += e * e;
    if (dp) dp[i] = 2.f * e / n;
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *loss = part[0] / n;
}

// g[j] = sum_i d[i, j]  (bias gradients)
__global__ void k_colsum(const float* __restrict__ d, float* __restrict__ g, int rows, int cols) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= cols) return;
  float s = 0.f;
  for (int i = 0; i < rows; ++i) s += d[(size_t)i * cols + j];
  g[j] = s;
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, int64_t n, float lr, float b1, float b2, float eps,
                       float c1, float c2, float wd) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float gi = g[i];
  float mi = b1 * m[i] + (1.f - b1) * gi;
  float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  // decoupled weight decay (AdamW): w <- w - lr * (mhat / (sqrt(vhat) + eps) + wd * w)
  w[i] -= lr * ((mi / c1) / (sqrtf(vi / c2) + eps) + wd * w[i]);
}

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

template <int TA, int TB>
void gemm(cudaStream_t s, const float* A, const float* B, float* C, const float* bias, int M, int N,
          int K, int relu, int accumulate) {
  dim3 grid((N + TN - 1) / TN, (M + TM - 1) / TM);
  k_gemm<TA, TB><<<grid, 256, 0, s>>>(A, B, C, bias, M, N, K, relu, accumulate);
  check(cudaGetLastError(), "mlp gemm launch");
}

}  // namespace

Mlp::Mlp(int in_dim, int hidden, int layers, uint64_t seed, cudaStream_t stream) : stream_(stream) {
  if (in_dim < 1 || hidden < 1 || layers < 1) throw std::invalid_argument("mlp: bad shape");
  dims_.push_back(in_dim);
  for (int l = 0; l < layers; ++l) dims_.push_back(hidden);
  dims_.push_back(1);
  for (size_t l = 0; l + 1 < dims_.size(); ++l) {
    woff_.push_back(n_params_);
    n_params_ += static_cast<int64_t>(dims_[l]) * dims_[l + 1];
    boff_.push_back(n_params_);
    n_params_ += dims_[l + 1];
  }
  // He initialisation, zero biases
  std::vector<float> h(n_params_, 0.f);
  std::mt19937_64 rng(seed);
  for (size_t l = 0; l + 1 < dims_.size(); ++l) {
    std::normal_distribution<float> nd(0.f, std::sqrt(2.f / dims_[l]));
    for (int64_t i = 0; i < static_cast<int64_t>(dims_[l]) * dims_[l + 1]; ++i) h[woff_[l] + i] = nd(rng);
  }
  const size_t bytes = static_cast<size_t>(n_params_) * 4;
  check(cudaMalloc(&w_, bytes), "mlp alloc");
  check(cudaMalloc(&g_, bytes), "mlp alloc");
  check(cudaMalloc(&m_, bytes), "mlp alloc");
  check(cudaMalloc(&v_, bytes), "mlp alloc");
  check(cudaMalloc(&loss_, 256), "mlp alloc");
  check(cudaMemcpyAsync(w_, h.data(), bytes, cudaMemcpyHostToDevice, stream_), "mlp init");
  check(cudaMemsetAsync(m_, 0, bytes, stream_), "mlp init");
  check(cudaMemsetAsync(v_, 0, bytes, stream_), "mlp init");
  check(cudaStreamSynchronize(stream_), "mlp init");
}

Mlp::~Mlp() {
  cudaStreamSynchronize(stream_);
  for (float* p : {w_, g_, m_, v_, x_, y_, loss_}) if (p) cudaFree(p);
  for (float* p : act_) cudaFree(p);
  for (float* p : delta_) cudaFree(p);
}

void Mlp::ensure(int n) {
  if (n <= cap_) return;
  cudaStreamSynchronize(stream_);
  for (float* p : act_) cudaFree(p);
  for (float* p : delta_) cudaFree(p);
  if (x_) cudaFree(x_);
  if (y_) cudaFree(y_);
  act_.clear();
  delta_.clear();
  cap_ = std::max(n, 256);
  check(cudaMalloc(&x_, static_cast<size_t>(cap_) * dims_[0] * 4), "mlp alloc");
  check(cudaMalloc(&y_, static_cast<size_t>(cap_) * 4), "mlp alloc");
  for (size_t l = 1; l < dims_.size(); ++l) {
    float *a = nullptr, *d = nullptr;
    check(cudaMalloc(&a, static_cast<size_t>(cap_) * dims_[l] * 4), "mlp alloc");
    check(cudaMalloc(&d, static_cast<size_t>(cap_) * dims_[l] * 4), "mlp alloc");
    act_.push_back(a);
    delta_.push_back(d);
  }
}

void Mlp::upload(const float* x, const float* y, int n) {
  ensure(n);
  check(cudaMemcpyAsync(x_, x, static_cast<size_t>(n) * dims_[0] * 4, cudaMemcpyHostToDevice, stream_),
        "mlp upload");
  if (y) check(cudaMemcpyAsync(y_, y, static_cast<size_t>(n) * 4, cudaMemcpyHostToDevice, stream_), "mlp upload");
}

void Mlp::forward(int n) {
  const int L = static_cast<int>(dims_.size()) - 1;
  for (int l = 0; l < L; ++l) {
    const float* in = l == 0 ? x_ : act_[l - 1];
    gemm<0, 0>(stream_, in, w_ + woff_[l], act_[l], w_ + boff_[l], n, dims_[l + 1], dims_[l],
               l + 1 < L ? 1 : 0, 0);
    ++launches;
  }
}

float Mlp::backward(int n) {
  const int L = static_cast<int>(dims_.size()) - 1;
  k_mse<<<1, 256, 0, stream_>>>(act_[L - 1], y_, delta_[L - 1], loss_, n);
  check(cudaGetLastError(), "mlp mse");
  for (int l = L - 1; l >= 0; --l) {
    const float* in = l == 0 ? x_ : act_[l - 1];
    // dW_l = in^T * delta_l ; db_l = colsum(delta_l)
    gemm<1, 0>(stream_, in, delta_[l], g_ + woff_[l], nullptr, dims_[l], dims_[l + 1], n, 0, 0);
    k_colsum<<<(dims_[l + 1] + 255) / 256, 256, 0, stream_>>>(delta_[l], g_ + boff_[l], n, dims_[l + 1]);
    if (l > 0) {
      // delta_{l-1} = (delta_l * W_l^T) .* relu'(act_{l-1})
      gemm<0, 1>(stream_, delta_[l], w_ + woff_[l], delta_[l - 1], nullptr, n, dims_[l], dims_[l + 1], 0, 0);
      int64_t cnt = static_cast<int64_t>(n) * dims_[l];
      k_relu_backward<<<static_cast<unsigned>((cnt + 255) / 256), 256, 0, stream_>>>(delta_[l - 1],
                                                                                      act_[l - 1], cnt);
    }
    launches += 3;
  }
  check(cudaGetLastError(), "mlp backward");
  float h = 0.f;
  check(cudaMemcpyAsync(&h, loss_, 4, cudaMemcpyDeviceToHost, stream_), "mlp loss");
  check(cudaStreamSynchronize(stream_), "mlp backward");
  return h;
}

float Mlp::train_step(const float* x, const float* y, int n, float lr) {
  upload(x, y, n);
  forward(n);
  float loss = backward(n);
  ++step_;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, static_cast<float>(step_));
  const float c2 = 1.f - std::pow(b2, static_cast<float>(step_));
  k_adam<<<static_cast<unsigned>((n_params_ + 255) / 256), 256, 0, stream_>>>(w_, g_, m_, v_, n_params_, lr,
                                                                                b1, b2, 1e-8f, c1, c2,
                                                                                weight_decay_);
  check(cudaGetLastError(), "mlp adam");
  ++launches;
  return loss;
}

void Mlp::predict(const float* x, int n, float* out) {
  upload(x, nullptr, n);
  forward(n);
  check(cudaMemcpyAsync(out, act_.back(), static_cast<size_t>(n) * 4, cudaMemcpyDeviceToHost, stream_),
        "mlp predict");
  check(cudaStreamSynchronize(stream_), "mlp predict");
}

float Mlp::gradients(const float* x, const float* y, int n, float* grad) {
  upload(x, y, n);
  forward(n);
  float loss = backward(n);
  check(cudaMemcpy(grad, g_, static_cast<size_t>(n_params_) * 4, cudaMemcpyDeviceToHost), "mlp grad");
  return loss;
}

void Mlp::get_params(float* out) const {
  check(cudaStreamSynchronize(stream_), "mlp params");
  check(cudaMemcpy(out, w_, static_cast<size_t>(n_params_) * 4, cudaMemcpyDeviceToHost), "mlp params");
}

void Mlp::set_params(const float* in) {
  check(cudaMemcpyAsync(w_, in, static_cast<size_t>(n_params_) * 4, cudaMemcpyHostToDevice, stream_),
        "mlp params");
  check(cudaMemsetAsync(m_, 0, static_cast<size_t>(n_params_) * 4, stream_), "mlp params");
  check(cudaMemsetAsync(v_, 0, static_cast<size_t>(n_params_) * 4, stream_), "mlp params");
  check(cudaStreamSynchronize(stream_), "mlp params");
  step_ = 0;
}

}  // namespace bsz
