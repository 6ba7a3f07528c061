// Warm-start network: an MLP (Fourier features of the cell centre (x, y)
// plus (m, p, t, Mach, AoA) -> 4 hidden layers of 256 SiLU units -> 8
// outputs: the 4 conserved variables and the 4 adjoint components, both
// normalised by the caller), trained and run on the GPU by this file's own
// kernels.  Every matrix product is the tcgen05 GEMM of mlp_gemm.cuh (BF16
// weights and activations, FP32 accumulation); biases, Adam moments and
// master weights are FP32.
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "mlp.hpp"
#include "mlp_gemm.cuh"

namespace o2f {
namespace mlp {

namespace {

constexpr int kIn = 7;         // x, y, m, p, t, Mach, AoA
constexpr int kFreq = 32;      // Fourier frequencies of (x, y)
constexpr int kFeat = 128;     // 2*kFreq sin/cos + kIn raw inputs, zero padded
constexpr int kWidth = 256;
constexpr int kHidden = 4;
constexpr int kOut = 8;
constexpr int kOutPad = 16;    // the output layer's GEMM tile width
constexpr int kSmemBytes = 100 * 1024;  // also caps residency at 2 CTAs (2 x 256 TMEM columns) per SM

int in_dim(int l) { return l == 0 ? kFeat : kWidth; }
int out_dim(int l) { return l == kHidden ? kOutPad : kWidth; }

__global__ void k_features(int n, const float* __restrict__ inputs, const int* __restrict__ index,
                           const float* __restrict__ freq, bf16* __restrict__ X) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* in = inputs + (int64_t)(index ? index[i] : i) * kIn;
  bf16* x = X + (int64_t)i * kFeat;
  const float px = in[0], py = in[1];
  for (int f = 0; f < kFreq; ++f) {
    const float arg = 6.283185307179586f * (freq[2 * f] * px + freq[2 * f + 1] * py);
    x[f] = __float2bfloat16_rn(sinf(arg));
    x[kFreq + f] = __float2bfloat16_rn(cosf(arg));
  }
  for (int j = 0; j < kIn; ++j) x[2 * kFreq + j] = __float2bfloat16_rn(in[j]);
  for (int j = 2 * kFreq + kIn; j < kFeat; ++j) x[j] = __float2bfloat16_rn(0.f);
}

// Mean squared error over the 8 outputs; dY = d(loss)/dY (bf16, padded
// columns zero); loss accumulated into *loss.
__global__ void k_loss(int n, const float* __restrict__ Y, const float* __restrict__ targets,
                       const int* __restrict__ index, bf16* __restrict__ dY, float* loss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  if (i < n) {
    const float* t = targets + (int64_t)(index ? index[i] : i) * kOut;
    const float scale = 2.f / ((float)n * kOut);
    for (int j = 0; j < kOutPad; ++j) {
      float g = 0.f;
      if (j < kOut) {
        const float d = Y[(int64_t)i * kOutPad + j] - t[j];
        l += d * d;
        g = scale * d;
      }
      dY[(int64_t)i * kOutPad + j] = __float2bfloat16_rn(g);
    }
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, l / ((float)n * kOut));
}

// db[j] += sum over rows of G(row, j)
__global__ void k_colsum(int n, int cols, const bf16* __restrict__ G, float* __restrict__ db) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= cols) return;
  const int rows_per = (n + gridDim.y - 1) / gridDim.y;
  const int r0 = blockIdx.y * rows_per, r1 = min(n, r0 + rows_per);
  float s = 0.f;
  for (int r = r0; r < r1; ++r) s += __bfloat162float(G[(int64_t)r * cols + j]);
  atomicAdd(db + j, s);
}

// Adam on the FP32 master parameters, then the BF16 copies of the weights in
// both orientations (W: [out][in] for the forward GEMM, WT: [in][out] for the
// input gradients).
__global__ void k_adam(int64_t n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

__global__ void k_pack(int rows, int cols, const float* __restrict__ w, bf16* __restrict__ W, bf16* __restrict__ WT) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)rows * cols) return;
  const int r = (int)(i / cols), c = (int)(i % cols);
  const bf16 b = __float2bfloat16_rn(w[i]);
  W[i] = b;
  WT[(int64_t)c * rows + r] = b;
}

int blocks_of(int64_t n, int b) { return (int)((n + b - 1) / b); }

}  // namespace

Mlp::Mlp(int max_batch, float freq_scale, uint64_t seed, cudaStream_t stream)
    : max_batch_(max_batch), stream_(stream) {
  if (max_batch < 128 || max_batch > (1 << 20)) throw Error(O2F_ERR_ARG, "max_batch out of range [128, 2^20]");
  if (!(freq_scale > 0.f)) throw Error(O2F_ERR_ARG, "freq_scale must be positive");
  O2F_CUDA(cudaFuncSetAttribute(k_gemm_tc<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes));
  O2F_CUDA(cudaFuncSetAttribute(k_gemm_tc<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes));
  // parameter layout: W0, b0, W1, b1, ..., W4, b4
  int64_t off = 0;
  for (int l = 0; l <= kHidden; ++l) {
    w_off_[l] = off;
    off += (int64_t)out_dim(l) * in_dim(l);
    b_off_[l] = off;
    off += out_dim(l);
  }
  n_params_ = off;
  std::mt19937_64 rng(seed);
  std::normal_distribution<float> nd(0.f, 1.f);
  std::vector<float> p(n_params_, 0.f);
  for (int l = 0; l <= kHidden; ++l) {
    const float s = std::sqrt(2.f / (float)in_dim(l)) * (l == kHidden ? 0.1f : 1.f);
    const int rows = l == kHidden ? kOut : out_dim(l);  // padded output rows stay zero
    for (int64_t i = 0; i < (int64_t)rows * in_dim(l); ++i) p[w_off_[l] + i] = s * nd(rng);
  }
  std::vector<float> fr(2 * kFreq);
  for (auto& f : fr) f = freq_scale * nd(rng);
  params_ = arena_.alloc<float>(n_params_);
  grads_ = arena_.alloc<float>(n_params_);
  adam_m_ = arena_.alloc<float>(n_params_);
  adam_v_ = arena_.alloc<float>(n_params_);
  freq_ = arena_.alloc<float>(2 * kFreq);
  for (int l = 0; l <= kHidden; ++l) {
    const int64_t n = (int64_t)out_dim(l) * in_dim(l);
    Wb_[l] = arena_.alloc<bf16>(n);
    WTb_[l] = arena_.alloc<bf16>(n);
  }
  X0_ = arena_.alloc<bf16>((int64_t)max_batch * kFeat);
  for (int l = 0; l < kHidden; ++l) {
    Z_[l] = arena_.alloc<bf16>((int64_t)max_batch * kWidth);
    A_[l] = arena_.alloc<bf16>((int64_t)max_batch * kWidth);
  }
  Y_ = arena_.alloc<float>((int64_t)max_batch * kOutPad);
  dY_ = arena_.alloc<bf16>((int64_t)max_batch * kOutPad);
  dZa_ = arena_.alloc<bf16>((int64_t)max_batch * kWidth);
  dZb_ = arena_.alloc<bf16>((int64_t)max_batch * kWidth);
  index_ = arena_.alloc<int>(max_batch);
  loss_ = arena_.alloc<float>(1);
  err_ = arena_.alloc<int>(1);
  O2F_CUDA(cudaMemcpyAsync(params_, p.data(), n_params_ * sizeof(float), cudaMemcpyHostToDevice, stream_));
  O2F_CUDA(cudaMemcpyAsync(freq_, fr.data(), fr.size() * sizeof(float), cudaMemcpyHostToDevice, stream_));
  O2F_CUDA(cudaMemsetAsync(adam_m_, 0, n_params_ * sizeof(float), stream_));
  O2F_CUDA(cudaMemsetAsync(adam_v_, 0, n_params_ * sizeof(float), stream_));
  O2F_CUDA(cudaMemsetAsync(err_, 0, sizeof(int), stream_));
  pack();
  sync();
}

void Mlp::sync() {
  O2F_CUDA(cudaStreamSynchronize(stream_));
  int e = 0;
  O2F_CUDA(cudaMemcpy(&e, err_, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    O2F_CUDA(cudaMemset(err_, 0, sizeof(int)));
    throw Error(O2F_ERR_CUDA, "tensor-core GEMM: an mbarrier wait exceeded its limit");
  }
}

void Mlp::pack() {
  for (int l = 0; l <= kHidden; ++l) {
    const int64_t n = (int64_t)out_dim(l) * in_dim(l);
    k_pack<<<blocks_of(n, 256), 256, 0, stream_>>>(out_dim(l), in_dim(l), params_ + w_off_[l], Wb_[l], WTb_[l]);
  }
  O2F_CUDA(cudaGetLastError());
}

void Mlp::gemm(int nt, const GemmArgs& a, int splits) {
  const dim3 grid(blocks_of(a.M, kTileM), blocks_of(a.N, nt), splits);
  if (nt == 256)
    k_gemm_tc<256><<<grid, kGemmThreads, kSmemBytes, stream_>>>(a);
  else
    k_gemm_tc<16><<<grid, kGemmThreads, kSmemBytes, stream_>>>(a);
  O2F_CUDA(cudaGetLastError());
  ++launches_;
}

GemmArgs Mlp::args() const {
  GemmArgs a{};
  a.err = err_;
  return a;
}

// Forward pass of n feature rows (X0_ filled): Z_/A_ per hidden layer, Y_.
void Mlp::forward(int n) {
  const bf16* x = X0_;
  for (int l = 0; l <= kHidden; ++l) {
    GemmArgs a = args();
    a.M = n;
    a.N = out_dim(l);
    a.K = in_dim(l);
    a.A = x;
    a.sam = in_dim(l);
    a.sak = 1;
    a.B = Wb_[l];
    a.sbn = in_dim(l);
    a.sbk = 1;
    a.k_split = a.K;
    a.bias = params_ + b_off_[l];
    if (l < kHidden) {
      a.epi = kEpiHidden;
      a.out = A_[l];
      a.pre = Z_[l];
      a.ldo = kWidth;
      gemm(256, a, 1);
      x = A_[l];
    } else {
      a.epi = kEpiLinear;
      a.out32 = Y_;
      a.ldo = kOutPad;
      gemm(16, a, 1);
    }
  }
}

// Backward pass from dY_ into grads_ (zeroed here).
void Mlp::backward(int n) {
  O2F_CUDA(cudaMemsetAsync(grads_, 0, n_params_ * sizeof(float), stream_));
  const bf16* g = dY_;  // gradient w.r.t. the output of layer l
  bf16* bufs[2] = {dZa_, dZb_};
  const int rows_split = 8;  // row slices of the bias column sums
  for (int l = kHidden; l >= 0; --l) {
    const int N = out_dim(l), K = in_dim(l);
    const bf16* below = l > 0 ? A_[l - 1] : X0_;
    // dW_l[n][k] = sum_m g(m, n) below(m, k): the batch is the reduction axis
    GemmArgs w = args();
    w.M = N;
    w.N = K;
    w.K = n;
    w.A = g;
    w.sam = 1;
    w.sak = N;
    w.B = below;
    w.sbn = 1;
    w.sbk = K;
    const int splits = std::max(1, std::min(64, (n + 2047) / 2048));
    w.k_split = ((n + splits - 1) / splits + kKC - 1) / kKC * kKC;
    w.epi = kEpiAtomic;
    w.out32 = grads_ + w_off_[l];
    w.ldo = K;
    gemm(256, w, (n + w.k_split - 1) / w.k_split);
    k_colsum<<<dim3(blocks_of(N, 128), rows_split), 128, 0, stream_>>>(n, N, g, grads_ + b_off_[l]);
    if (l == 0) break;
    // gradient w.r.t. the layer below's pre-activation: (g W_l) * silu'(Z_{l-1})
    GemmArgs d = args();
    d.M = n;
    d.N = K;
    d.K = N;
    d.A = g;
    d.sam = N;
    d.sak = 1;
    d.B = WTb_[l];
    d.sbn = N;
    d.sbk = 1;
    d.k_split = d.K;
    d.epi = kEpiBackAct;
    bf16* out = bufs[l & 1];
    d.out = out;
    d.zprev = Z_[l - 1];
    d.ldo = kWidth;
    gemm(256, d, 1);
    g = out;
  }
  O2F_CUDA(cudaGetLastError());
}

void Mlp::load_batch(const float* inputs_dev, const int* index_dev, int n) {
  k_features<<<blocks_of(n, 128), 128, 0, stream_>>>(n, inputs_dev, index_dev, freq_, X0_);
  O2F_CUDA(cudaGetLastError());
}

void Mlp::set_data(const float* inputs, const float* targets, int64_t n) {
  if (n <= 0) throw Error(O2F_ERR_ARG, "empty data set");
  if (n > data_cap_) {  // device buffers grow only: repeated calls reuse them
    data_in_ = arena_.alloc<float>(n * kIn);
    data_out_ = arena_.alloc<float>(n * kOut);
    data_cap_ = n;
  }
  n_data_ = n;
  O2F_CUDA(cudaMemcpyAsync(data_in_, inputs, n * kIn * sizeof(float), cudaMemcpyHostToDevice, stream_));
  O2F_CUDA(cudaMemcpyAsync(data_out_, targets, n * kOut * sizeof(float), cudaMemcpyHostToDevice, stream_));
  sync();
}

void Mlp::train(int steps, int batch, float lr, uint64_t seed, float* loss_hist) {
  if (!n_data_) throw Error(O2F_ERR_STATE, "no training data (o2f_mlp_set_data)");
  if (steps <= 0 || batch < 1 || batch > max_batch_) throw Error(O2F_ERR_ARG, "steps or batch out of range");
  if (!(lr > 0.f)) throw Error(O2F_ERR_ARG, "lr must be positive");
  std::mt19937_64 rng(seed);
  std::uniform_int_distribution<int64_t> pick(0, n_data_ - 1);
  std::vector<int> idx(batch);
  if (steps > loss_cap_) {
    loss_buf_ = arena_.alloc<float>(steps);
    loss_cap_ = steps;
  }
  float* losses = loss_buf_;
  O2F_CUDA(cudaMemsetAsync(losses, 0, steps * sizeof(float), stream_));
  int* pinned = nullptr;
  O2F_CUDA(cudaMallocHost(&pinned, sizeof(int) * batch));
  try {
    for (int s = 0; s < steps; ++s) {
      for (int i = 0; i < batch; ++i) idx[i] = (int)pick(rng);
      O2F_CUDA(cudaStreamSynchronize(stream_));  // the pinned index buffer is free again
      std::memcpy(pinned, idx.data(), sizeof(int) * batch);
      O2F_CUDA(cudaMemcpyAsync(index_, pinned, sizeof(int) * batch, cudaMemcpyHostToDevice, stream_));
      load_batch(data_in_, index_, batch);
      forward(batch);
      k_loss<<<blocks_of(batch, 128), 128, 0, stream_>>>(batch, Y_, data_out_, index_, dY_, losses + s);
      backward(batch);
      ++adam_t_;
      const float b1 = 0.9f, b2 = 0.999f;
      const float c1 = 1.f - std::pow(b1, (float)adam_t_), c2 = 1.f - std::pow(b2, (float)adam_t_);
      k_adam<<<blocks_of(n_params_, 256), 256, 0, stream_>>>(n_params_, params_, grads_, adam_m_, adam_v_, lr, b1,
                                                             b2, 1e-8f, c1, c2);
      pack();
    }
    sync();
  } catch (...) {
    cudaFreeHost(pinned);
    throw;
  }
  cudaFreeHost(pinned);
  if (loss_hist) O2F_CUDA(cudaMemcpy(loss_hist, losses, steps * sizeof(float), cudaMemcpyDeviceToHost));
}

void Mlp::predict(const float* inputs, int64_t n, float* out) {
  if (n <= 0) return;
  float* in_dev = arena_scratch_in(n);
  O2F_CUDA(cudaMemcpyAsync(in_dev, inputs, n * kIn * sizeof(float), cudaMemcpyHostToDevice, stream_));
  std::vector<float> y((size_t)max_batch_ * kOutPad);
  for (int64_t b0 = 0; b0 < n; b0 += max_batch_) {
    const int m = (int)std::min<int64_t>(max_batch_, n - b0);
    load_batch(in_dev + b0 * kIn, nullptr, m);
    forward(m);
    O2F_CUDA(cudaMemcpyAsync(y.data(), Y_, (size_t)m * kOutPad * sizeof(float), cudaMemcpyDeviceToHost, stream_));
    sync();
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < kOut; ++j) out[(b0 + i) * kOut + j] = y[(size_t)i * kOutPad + j];
  }
}

float* Mlp::arena_scratch_in(int64_t n) {
  if (scratch_cap_ < n) {
    scratch_in_ = arena_.alloc<float>(n * kIn);
    scratch_cap_ = n;
  }
  return scratch_in_;
}

void Mlp::gradients(const float* inputs, const float* targets, int n, float* grads_out, float* loss_out) {
  if (n < 1 || n > max_batch_) throw Error(O2F_ERR_ARG, "n out of range");
  float* in_dev = arena_scratch_in(n);
  if (!grad_targets_) grad_targets_ = arena_.alloc<float>((int64_t)max_batch_ * kOut);
  O2F_CUDA(cudaMemcpyAsync(in_dev, inputs, (size_t)n * kIn * sizeof(float), cudaMemcpyHostToDevice, stream_));
  O2F_CUDA(cudaMemcpyAsync(grad_targets_, targets, (size_t)n * kOut * sizeof(float), cudaMemcpyHostToDevice, stream_));
  O2F_CUDA(cudaMemsetAsync(loss_, 0, sizeof(float), stream_));
  load_batch(in_dev, nullptr, n);
  forward(n);
  k_loss<<<blocks_of(n, 128), 128, 0, stream_>>>(n, Y_, grad_targets_, nullptr, dY_, loss_);
  backward(n);
  sync();
  O2F_CUDA(cudaMemcpy(grads_out, grads_, n_params_ * sizeof(float), cudaMemcpyDeviceToHost));
  if (loss_out) O2F_CUDA(cudaMemcpy(loss_out, loss_, sizeof(float), cudaMemcpyDeviceToHost));
}

void Mlp::get_params(float* out, float* freq_out) {
  sync();
  O2F_CUDA(cudaMemcpy(out, params_, n_params_ * sizeof(float), cudaMemcpyDeviceToHost));
  if (freq_out) O2F_CUDA(cudaMemcpy(freq_out, freq_, 2 * kFreq * sizeof(float), cudaMemcpyDeviceToHost));
}

void Mlp::set_params(const float* in) {
  O2F_CUDA(cudaMemcpyAsync(params_, in, n_params_ * sizeof(float), cudaMemcpyHostToDevice, stream_));
  pack();
  sync();
}

}  // namespace mlp
}  // namespace o2f
