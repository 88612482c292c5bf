// FP32 MLP for the schedule cost model (see mlp.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace bsz {

class Mlp {
 public:
  Mlp(int in_dim, int hidden, int layers, uint64_t seed, cudaStream_t stream);
  ~Mlp();
  Mlp(const Mlp&) = delete;
  Mlp& operator=(const Mlp&) = delete;

  int64_t n_params() const { return n_params_; }
  // One Adam step on a batch (x: n x in_dim row-major, y: n); returns the loss
  // before the step.
  float train_step(const float* x, const float* y, int n, float lr);
  void predict(const float* x, int n, float* out);
  // Loss and gradient of the loss w.r.t. the flat parameters (no update).
  float gradients(const float* x, const float* y, int n, float* grad);
  void get_params(float* out) const;
  void set_weight_decay(float wd) { weight_decay_ = wd; }
  void set_params(const float* in);
  int64_t launches = 0;

 private:
  std::vector<int> dims_;
  std::vector<int64_t> woff_, boff_;
  int64_t n_params_ = 0;
  float* w_ = nullptr;
  float* g_ = nullptr;
  float* m_ = nullptr;
  float* v_ = nullptr;
  float* x_ = nullptr;
  float* y_ = nullptr;
  float* loss_ = nullptr;
  std::vector<float*> act_, delta_;
  int cap_ = 0;
  int64_t step_ = 0;
  float weight_decay_ = 0.f;
  cudaStream_t stream_;
  void ensure(int n);
  void upload(const float* x, const float* y, int n);
  void forward(int n);
  float backward(int n);
};

}  // namespace bsz
