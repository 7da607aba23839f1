// learned_io.cu -- between the Poisson unknown grid (FP64, (nky+1) rows of
// (nkx+1)) and the network's padded NHWC tensors (FP32, h x w, h and w
// multiples of 8, zero padding).
#include <cuda_runtime.h>

#include <cmath>

#include "device.hpp"
#include "kernels.hpp"
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

// The Poisson operator on the unknown grid (Dirichlet values folded into the
// right-hand side, so neighbours beyond a Dirichlet end are zero; periodic
// ends wrap), v(i, j) returning the entry at column i, row j.
template <class T, class V>
__device__ __forceinline__ T apply_op(const kern::PoissonLayout& L, int i, int j, int mx, int my, V v) {
  T a = T(L.Cd) * v(i, j);
  if (i > 0) a += T(L.Cx) * v(i - 1, j); else if (L.periodic_x) a += T(L.Cx) * v(mx - 1, j);
  if (i < mx - 1) a += T(L.Cx) * v(i + 1, j); else if (L.periodic_x) a += T(L.Cx) * v(0, j);
  if (j > 0) a += T(L.Cy) * v(i, j - 1); else if (L.periodic_y) a += T(L.Cy) * v(i, my - 1);
  if (j < my - 1) a += T(L.Cy) * v(i, j + 1); else if (L.periodic_y) a += T(L.Cy) * v(i, 0);
  return a;
}

__device__ __forceinline__ void block_add(double v, double* dst) {
  __shared__ double sh[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int q = 0; q < int(blockDim.x >> 5); ++q) t += sh[q];
    atomicAdd(dst, t);
  }
}

// in = b - A phi in FP64, stored as float on the padded grid; sum2 += r^2
__global__ void k_residual(const double* b, const double* phi, kern::PoissonLayout L, int h, int w, float* in,
                           double* sum2) {
  const int mx = L.nkx + 1, my = L.nky + 1;
  const size_t n = size_t(h) * w;
  double s = 0.0;
  for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x) {
    const int i = int(e % w), j = int(e / w);
    float v = 0.0f;
    if (i < mx && j < my) {
      const double r = b[size_t(i) + size_t(j) * mx] -
                       apply_op<double>(L, i, j, mx, my, [&](int a, int c) { return phi[size_t(a) + size_t(c) * mx]; });
      v = float(r);
      s += r * r;
    }
    in[e] = v;
  }
  block_add(s, sum2);
}

// in /= s with s = RMS of the residual over the unknowns; scale[0] = s
__global__ void k_normalise(float* in, size_t n, const double* sum2, int nvalid, float* scale) {
  const double rms = sqrt(sum2[0] / double(nvalid));
  const float inv = rms > 0 ? float(1.0 / rms) : 0.0f;
  if (blockIdx.x == 0 && threadIdx.x == 0) scale[0] = float(rms);
  for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x)
    in[e] *= inv;
}

// x = prev + out * s / |Cd| (out: the correction in units of the residual's
// RMS divided by the operator's diagonal)
__global__ void k_apply_residual(const float* out, const double* prev, int mx, int my, int w, const float* scale,
                                 double inv_cd, double* x) {
  const size_t n = size_t(mx) * my;
  const double f = double(scale[0]) * inv_cd;
  for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x) {
    const int i = int(k % mx), j = int(k / mx);
    x[k] = prev[k] + double(out[size_t(j) * w + i]) * f;
  }
}

// res = in - (A / |Cd|) out on the unknowns (zero on the padding); loss += mean res^2
__global__ void k_res_loss(const float* out, const float* in, kern::PoissonLayout L, float inv_cd, int h, int w,
                           float* res, double* loss) {
  const int mx = L.nkx + 1, my = L.nky + 1;
  const size_t n = size_t(h) * w;
  double s = 0.0;
  for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x) {
    const int i = int(e % w), j = int(e / w);
    float v = 0.0f;
    if (i < mx && j < my) {
      v = in[e] - inv_cd * apply_op<float>(L, i, j, mx, my, [&](int a, int c) { return out[size_t(c) * w + a]; });
      s += double(v) * v;
    }
    res[e] = v;
  }
  block_add(s / double(mx * my), loss);
}

// g = d(mean res^2)/d out = -2 (A / |Cd|)^T res / n (A symmetric: Dirichlet
// and periodic ends only)
__global__ void k_res_grad(const float* res, kern::PoissonLayout L, float inv_cd, int h, int w, float* g) {
  const int mx = L.nkx + 1, my = L.nky + 1;
  const size_t n = size_t(h) * w;
  const float f = -2.0f * inv_cd / float(mx * my);
  for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x) {
    const int i = int(e % w), j = int(e / w);
    g[e] = (i < mx && j < my)
               ? f * apply_op<float>(L, i, j, mx, my, [&](int a, int c) { return res[size_t(c) * w + a]; })
               : 0.0f;
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

void residual_input(const double* b, const double* phi, const kern::PoissonLayout& L, int h, int w, float* in,
                    double* sum2, float* scale, cudaStream_t s) {
  GP_CUDA(cudaMemsetAsync(sum2, 0, sizeof(double), s));
  const size_t n = size_t(h) * w;
  k_residual<<<grid_for(n), 256, 0, s>>>(b, phi, L, h, w, in, sum2);
  GP_LAUNCH_CHECK();
  k_normalise<<<grid_for(n), 256, 0, s>>>(in, n, sum2, (L.nkx + 1) * (L.nky + 1), scale);
  GP_LAUNCH_CHECK();
}

void apply_residual_correction(const float* out, const double* prev, const kern::PoissonLayout& L, int w,
                               const float* scale, double* x, cudaStream_t s) {
  const int mx = L.nkx + 1, my = L.nky + 1;
  k_apply_residual<<<grid_for(size_t(mx) * my), 256, 0, s>>>(out, prev, mx, my, w, scale, 1.0 / std::fabs(L.Cd), x);
  GP_LAUNCH_CHECK();
}

void residual_loss_grad(const float* out, const float* in, const kern::PoissonLayout& L, int h, int w, float* res,
                        float* g, double* loss, cudaStream_t s) {
  const float inv_cd = float(1.0 / std::fabs(L.Cd));
  const size_t n = size_t(h) * w;
  k_res_loss<<<grid_for(n), 256, 0, s>>>(out, in, L, inv_cd, h, w, res, loss);
  GP_LAUNCH_CHECK();
  k_res_grad<<<grid_for(n), 256, 0, s>>>(res, L, inv_cd, h, w, g);
  GP_LAUNCH_CHECK();
}

}  // namespace nn
}  // namespace gample
