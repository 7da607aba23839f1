// learned_io.cu -- between the Poisson unknown grid (FP64, (nky+1) rows of
// (nkx+1)) and the network's padded NHWC tensors (FP32, h x w, h and w
// multiples of 8, zero padding).
#include <cuda_runtime.h>

#include "device.hpp"
#include "learned.hpp"

namespace gample {
namespace nn {

namespace {

int grid_for(size_t n) {
  const size_t b = (n + 255) / 256;
  return int(b < 148 * 8 ? (b ? b : 1) : 148 * 8);
}

// scale[0..2] = 1 / RMS of b, of phi and of the last correction (device)
__global__ void k_pack(const double* b, const double* phi, int mx, int my, int h, int w, const float* inv, float* in) {
  const size_t n = size_t(h) * w;
  for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x) {
    const int i = int(e % w), j = int(e / w);
    float v0 = 0.0f, v1 = 0.0f;
    if (i < mx && j < my) {
      const size_t k = size_t(i) + size_t(j) * mx;
      v0 = float(b[k] * inv[0]);
      v1 = float(phi[k] * inv[1]);
    }
    in[2 * e] = v0;
    in[2 * e + 1] = v1;
  }
}

// x = prev + out / inv[2]
__global__ void k_apply(const float* out, const double* prev, int mx, int my, int w, const float* inv, double* x) {
  const size_t n = size_t(mx) * my;
  const double s = 1.0 / double(inv[2]);
  for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x) {
    const int i = int(k % mx), j = int(k / mx);
    x[k] = prev[k] + double(out[size_t(j) * w + i]) * s;
  }
}

// target = (x - prev) * inv[2]; sums[0..2] += sum b^2, phi^2, (x - prev)^2
__global__ void k_target(const double* x, const double* prev, const double* b, int mx, int my, int h, int w,
                         const float* inv, float* target, double* sums) {
  __shared__ double sh[3][32];
  const size_t n = size_t(h) * w;
  double s0 = 0, s1 = 0, s2 = 0;
  for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x) {
    const int i = int(e % w), j = int(e / w);
    float t = 0.0f;
    if (i < mx && j < my) {
      const size_t k = size_t(i) + size_t(j) * mx;
      const double d = x[k] - prev[k];
      t = float(d * inv[2]);
      s0 += b[k] * b[k];
      s1 += x[k] * x[k];
      s2 += d * d;
    }
    target[e] = t;
  }
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    sh[0][wid] = s0;
    sh[1][wid] = s1;
    sh[2][wid] = s2;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0;
    for (int q = 0; q < int(blockDim.x >> 5); ++q) t += sh[threadIdx.x][q];
    atomicAdd(sums + threadIdx.x, t);
  }
}

}  // namespace

void pack_input(const double* b, const double* phi, int mx, int my, int h, int w, const float* inv, float* in,
                cudaStream_t s) {
  k_pack<<<grid_for(size_t(h) * w), 256, 0, s>>>(b, phi, mx, my, h, w, inv, in);
  GP_LAUNCH_CHECK();
}

void apply_correction(const float* out, const double* prev, int mx, int my, int w, const float* inv, double* x,
                      cudaStream_t s) {
  k_apply<<<grid_for(size_t(mx) * my), 256, 0, s>>>(out, prev, mx, my, w, inv, x);
  GP_LAUNCH_CHECK();
}

void make_target(const double* x, const double* prev, const double* b, int mx, int my, int h, int w,
                 const float* inv, float* target, double* sums, cudaStream_t s) {
  GP_CUDA(cudaMemsetAsync(sums, 0, 3 * sizeof(double), s));
  k_target<<<grid_for(size_t(h) * w), 256, 0, s>>>(x, prev, b, mx, my, h, w, inv, target, sums);
  GP_LAUNCH_CHECK();
}

}  // namespace nn
}  // namespace gample
