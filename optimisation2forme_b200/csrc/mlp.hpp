// Warm-start network (mlp.cu): host driver of the tcgen05 training and
// inference kernels.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

#include "solver.hpp"

namespace o2f {
namespace mlp {

struct GemmArgs;

class Mlp {
 public:
  Mlp(int max_batch, float freq_scale, uint64_t seed, cudaStream_t stream);
  int64_t n_params() const { return n_params_; }
  void set_data(const float* inputs, const float* targets, int64_t n);
  void train(int steps, int batch, float lr, uint64_t seed, float* loss_hist);
  void predict(const float* inputs, int64_t n, float* out);
  void gradients(const float* inputs, const float* targets, int n, float* grads_out, float* loss_out);
  void get_params(float* out, float* freq_out);
  void set_params(const float* in);
  int64_t launches() const { return launches_; }

 private:
  void sync();
  void pack();
  void gemm(int nt, const GemmArgs& a, int splits);
  GemmArgs args() const;
  void forward(int n);
  void backward(int n);
  void load_batch(const float* inputs_dev, const int* index_dev, int n);
  float* arena_scratch_in(int64_t n);

  int max_batch_;
  cudaStream_t stream_;
  DeviceArena arena_;
  int64_t n_params_ = 0;
  int64_t w_off_[5]{}, b_off_[5]{};
  float *params_ = nullptr, *grads_ = nullptr, *adam_m_ = nullptr, *adam_v_ = nullptr, *freq_ = nullptr;
  __nv_bfloat16 *Wb_[5]{}, *WTb_[5]{};
  __nv_bfloat16* X0_ = nullptr;
  __nv_bfloat16 *Z_[4]{}, *A_[4]{};
  float* Y_ = nullptr;
  __nv_bfloat16 *dY_ = nullptr, *dZa_ = nullptr, *dZb_ = nullptr;
  int* index_ = nullptr;
  float* loss_ = nullptr;
  int* err_ = nullptr;
  float *data_in_ = nullptr, *data_out_ = nullptr;
  int64_t n_data_ = 0, data_cap_ = 0;
  float* loss_buf_ = nullptr;
  int64_t loss_cap_ = 0;
  float* scratch_in_ = nullptr;
  int64_t scratch_cap_ = 0;
  float* grad_targets_ = nullptr;
  int64_t adam_t_ = 0;
  int64_t launches_ = 0;
};

}  // namespace mlp
}  // namespace o2f
