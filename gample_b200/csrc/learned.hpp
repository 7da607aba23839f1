// learned.hpp -- learned warm start of the Poisson solve.
//
// A 4-level convolutional encoder-decoder (3 x 3 kernels, 32/64/128/256
// channels, skip connections, BF16 weights and activations, FP32
// accumulation on the tensor cores) maps the normalised right-hand side and
// the previous solution on the unknown grid to a correction of the previous
// solution; the multigrid then solves from (previous + correction) to the
// same relative residual as without it, so the network only changes the
// starting point, never the answer. Training runs on the GPU with the same
// kernels (im2col + tcgen05 GEMM forward, GEMM-based input and weight
// gradients, Adam) on (rhs, previous phi) -> (phi - previous phi) pairs the
// simulator produces while it runs.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "device.hpp"
#include "kernels.hpp"

namespace gample {
namespace nn {

// out[row * ldo + n] = act(alpha * acc + bias[n]) for row < m_valid, n < n_valid
struct GemmEpilogue {
  float alpha = 1.0f;
  const float* bias = nullptr;
  int relu = 0;
  int accumulate = 0;  // out_f32 += value
  float* out_f32 = nullptr;
  __nv_bfloat16* out_bf16 = nullptr;
  int ldo = 0;
  int m_valid = 0, n_valid = 0;
  int split_k = 0;  // allow splitting K over CTAs (plain FP32 output, zeroed and accumulated atomically)
};

// Implicit im2col for A: row m = pixel m of an h x w NHWC tensor x with cin
// channels, column k = tap * cin + channel of the 3 x 3 neighbourhood (zero
// outside the grid). Needs K = 9 cin and cin a multiple of the K step.
struct ConvA {
  const __nv_bfloat16* x = nullptr;
  int h = 0, w = 0, cin = 0;
};

// C = A[M x K] * B[N x K]^T on the tensor cores (both K-major BF16); M a
// multiple of 128, N of 32, K of 32. err: device int set to 1 if an MMA
// completion wait timed out.
void gemm_bf16(const __nv_bfloat16* A, const __nv_bfloat16* B, int M, int N, int K, const GemmEpilogue& ep, int* err,
               cudaStream_t s, const ConvA& conv = ConvA{});

// Unknown grid <-> network tensors (inv: device floats 1/RMS of the rhs, of
// phi and of the correction).
void pack_input(const double* b, const double* phi, int mx, int my, int h, int w, const float* inv, float* in,
                cudaStream_t s);
void apply_correction(const float* out, const double* prev, int mx, int my, int w, const float* inv, double* x,
                      cudaStream_t s);
void make_target(const double* x, const double* prev, const double* b, int mx, int my, int h, int w,
                 const float* inv, float* target, double* sums, cudaStream_t s);

// Residual formulation of the warm start: in = (b - A phi) / s on the padded
// grid with s its RMS over the unknowns (scale[0] = s, sum2: one device
// double of scratch); x = prev + out * s / |Cd|; the loss of a correction
// out is mean((in - (A / |Cd|) out)^2) over the unknowns, whose gradient
// with respect to out is written to g (res: scratch of h * w floats, loss:
// one device double, accumulated).
void residual_input(const double* b, const double* phi, const kern::PoissonLayout& L, int h, int w, float* in,
                    double* sum2, float* scale, cudaStream_t s);
void apply_residual_correction(const float* out, const double* prev, const kern::PoissonLayout& L, int w,
                               const float* scale, double* x, cudaStream_t s);
void residual_loss_grad(const float* out, const float* in, const kern::PoissonLayout& L, int h, int w, float* res,
                        float* g, double* loss, cudaStream_t s);

struct ConvLayer {
  int cin, cout;           // channels
  int kpad;                // 9 * cin rounded up to a multiple of 32
  int cout_p;              // cout rounded up to a multiple of 32
  bool relu;
  DeviceArray<float> w, b;           // FP32 master weights [cout][kpad] (zero padding), bias
  DeviceArray<__nv_bfloat16> wb;     // BF16 copy [cout_p][kpad]
  DeviceArray<__nv_bfloat16> wt;     // BF16 transpose [kpad][cout_p] (input-gradient GEMM)
  DeviceArray<float> gw, gb;         // gradients
  DeviceArray<float> mw, vw, mb, vb; // Adam moments
};

class WarmStartNet {
 public:
  // h, w: grid (multiples of 8); the levels run at h, h/2, h/4, h/8 with
  // widths c[0..3]; cin0 input channels.
  WarmStartNet(int h, int w, uint64_t seed, cudaStream_t s, int cin0 = 2, const int (&c)[4] = kWideWidths);
  static constexpr int kWideWidths[4] = {32, 64, 128, 256};
  // in: NHWC input [h][w][cin0] FP32 (normalised); out: [h][w] FP32
  void forward(const float* in, float* out);
  int input_channels() const { return cin0_; }
  // One Adam step on the mean-squared error against target [h][w]; returns
  // the loss of the forward pass (synchronous read of one float).
  float train_step(const float* in, const float* target, float lr);
  // The same on the residual loss of a one-channel network (input: a
  // normalised residual, residual_input): the mean square of the residual
  // left by the correction the network predicts.
  float train_step_residual(const float* in, const kern::PoissonLayout& L, float lr);
  float loss_and_grad_residual(const float* in, const kern::PoissonLayout& L);
  // Parameter access for the gradient check (FP32 masters, layer by layer).
  int num_layers() const { return int(layers_.size()); }
  ConvLayer& layer(int i) { return layers_[i]; }
  void sync_weights();  // refresh the BF16 copies after the FP32 masters changed
  // forward + backward without the optimiser step (gradients left in gw/gb)
  float loss_and_grad(const float* in, const float* target);
  double flops_forward() const;
  int h() const { return h_; }
  int w() const { return w_; }
  cudaStream_t stream;

 private:
  struct Act {  // one activation tensor NHWC
    int h, w, c;
    DeviceArray<__nv_bfloat16> y;  // BF16 values (post activation)
    DeviceArray<float> g;          // FP32 gradient
  };
  void conv_forward(ConvLayer& L, const Act& x, Act& y, float* out_f32 = nullptr);
  void conv_backward(ConvLayer& L, const Act& x, Act& y, Act* dx, const float* gy_override = nullptr);
  void im2col(const Act& x, int kpad, int rows);  // into col_
  void backward(const float* gout);  // gradients of every layer from the output gradient
  void adam(float lr);               // one Adam step on the gradients, then the BF16 copies
  int h_, w_, cin0_;
  std::vector<ConvLayer> layers_;
  std::vector<Act> acts_;
  DeviceArray<__nv_bfloat16> col_, colT_, gyT_, gyb_;
  DeviceArray<float> gcol_, out_, gout_, loss_, res_;
  DeviceArray<double> lossd_;
  DeviceArray<int> err_;
  int step_ = 0;
};

}  // namespace nn
}  // namespace gample
