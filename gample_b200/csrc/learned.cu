// learned.cu -- the warm-start network: layers, forward, backward, Adam.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <random>
#include <stdexcept>

#include "learned.hpp"

namespace gample {
namespace nn {

namespace {

constexpr int kT = 256;

int grid_for(size_t n) {
  const size_t b = (n + kT - 1) / kT;
  return int(b < 148 * 16 ? (b ? b : 1) : 148 * 16);
}
int rup(int v, int m) { return (v + m - 1) / m * m; }

// Xcol[p][t * C + c] = X[p + offset(t)][c] (zero outside the grid and in the
// padding columns k >= 9C, rows p >= hw).
__global__ void k_im2col(const __nv_bfloat16* x, int h, int w, int c, int kpad, int rows, __nv_bfloat16* col) {
  const size_t n = size_t(rows) * kpad;
  for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x) {
    const int p = int(e / kpad), k = int(e % kpad);
    __nv_bfloat16 v = __float2bfloat16_rn(0.0f);
    if (p < h * w && k < 9 * c) {
      const int t = k / c, ch = k % c;
      const int yy = p / w + t / 3 - 1, xx = p % w + t % 3 - 1;
      if (yy >= 0 && yy < h && xx >= 0 && xx < w) v = x[(size_t(yy) * w + xx) * c + ch];
    }
    col[e] = v;
  }
}

// The same with 16-byte chunks of 8 channels (C a multiple of 8).
__global__ void k_im2col8(const __nv_bfloat16* x, int h, int w, int c, int kpad, int rows, __nv_bfloat16* col) {
  const int kc = kpad / 8;
  const size_t n = size_t(rows) * kc;
  for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x) {
    const int p = int(e / kc), k = int(e % kc) * 8;
    uint4 v = make_uint4(0, 0, 0, 0);
    if (p < h * w && k < 9 * c) {
      const int t = k / c, ch = k - t * c;
      const int yy = p / w + t / 3 - 1, xx = p % w + t % 3 - 1;
      if (yy >= 0 && yy < h && xx >= 0 && xx < w)
        v = *reinterpret_cast<const uint4*>(x + (size_t(yy) * w + xx) * c + ch);
    }
    *reinterpret_cast<uint4*>(col + size_t(p) * kpad + k) = v;
  }
}

// dX[q][c] += sum over taps t of dXcol[q - offset(t)][t * C + c]
__global__ void k_col2im_add(const float* gcol, int h, int w, int c, int kpad, float* gx) {
  const size_t n = size_t(h) * w * c;
  for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x) {
    const int q = int(e / c), ch = int(e % c);
    const int qy = q / w, qx = q % w;
    float s = 0.0f;
#pragma unroll
    for (int t = 0; t < 9; ++t) {
      const int py = qy - (t / 3 - 1), px = qx - (t % 3 - 1);
      if (py >= 0 && py < h && px >= 0 && px < w) s += gcol[(size_t(py) * w + px) * kpad + t * c + ch];
    }
    gx[e] += s;
  }
}

// dst[j][i] = src[i][j] (src rows x cols), zero-padded to dst_rows x dst_cols
__global__ void k_transpose(const __nv_bfloat16* src, int rows, int cols, int src_ld, __nv_bfloat16* dst,
                            int dst_rows, int dst_cols) {
  __shared__ __nv_bfloat16 tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;  // bx over src cols (dst rows), by over src rows
  for (int yy = threadIdx.y; yy < 32; yy += 8) {
    const int r = by + yy, cc = bx + threadIdx.x;
    tile[yy][threadIdx.x] = (r < rows && cc < cols) ? src[size_t(r) * src_ld + cc] : __float2bfloat16_rn(0.0f);
  }
  __syncthreads();
  for (int yy = threadIdx.y; yy < 32; yy += 8) {
    const int dr = bx + yy, dc = by + threadIdx.x;
    if (dr < dst_rows && dc < dst_cols) dst[size_t(dr) * dst_cols + dc] = tile[threadIdx.x][yy];
  }
}

// gy (pre-activation) = g * (y > 0 if relu); written as BF16 [rows][cout_p]
// (zero padding) and accumulated into the bias gradient.
__global__ void k_act_back(const float* g, const __nv_bfloat16* y, int hw, int c, int cout_p, int rows, int relu,
                           __nv_bfloat16* gyb, float* gb) {
  __shared__ float sb[256];
  for (int i = threadIdx.x; i < c; i += blockDim.x) sb[i] = 0.0f;
  __syncthreads();
  const size_t n = size_t(rows) * cout_p;
  for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x) {
    const int p = int(e / cout_p), ch = int(e % cout_p);
    float v = 0.0f;
    if (p < hw && ch < c) {
      v = g[size_t(p) * c + ch];
      if (relu && !(__bfloat162float(y[size_t(p) * c + ch]) > 0.0f)) v = 0.0f;
      atomicAdd(&sb[ch], v);
    }
    gyb[e] = __float2bfloat16_rn(v);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < c; i += blockDim.x)
    if (sb[i] != 0.0f) atomicAdd(gb + i, sb[i]);
}

__global__ void k_pool(const __nv_bfloat16* x, int h, int w, int c, __nv_bfloat16* y) {
  const int h2 = h / 2, w2 = w / 2;
  const size_t n = size_t(h2) * w2 * c;
  for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x) {
    const int ch = int(e % c), q = int(e / c), qy = q / w2, qx = q % w2;
    float s = 0.0f;
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b) s += __bfloat162float(x[((size_t(2 * qy + a)) * w + 2 * qx + b) * c + ch]);
    y[e] = __float2bfloat16_rn(0.25f * s);
  }
}

__global__ void k_pool_back(const float* gy, int h, int w, int c, float* gx) {
  const size_t n = size_t(h) * w * c;
  for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x) {
    const int ch = int(e % c), p = int(e / c), py = p / w, px = p % w;
    gx[e] += 0.25f * gy[(size_t(py / 2) * (w / 2) + px / 2) * c + ch];
  }
}

// Nearest upsampling of x [h/2][w/2][cx] into channels [0, cx) of y [h][w][cy]
// and a copy of s [h][w][cs] into channels [cx, cx + cs).
__global__ void k_up_concat(const __nv_bfloat16* x, int cx, const __nv_bfloat16* s, int cs, int h, int w,
                            __nv_bfloat16* y) {
  const int cy = cx + cs;
  const size_t n = size_t(h) * w * cy;
  for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x) {
    const int ch = int(e % cy), p = int(e / cy), py = p / w, px = p % w;
    y[e] = ch < cx ? x[(size_t(py / 2) * (w / 2) + px / 2) * cx + ch] : s[size_t(p) * cs + (ch - cx)];
  }
}

__global__ void k_up_concat_back(const float* gy, int cx, int cs, int h, int w, float* gx, float* gs) {
  const int cy = cx + cs;
  const size_t n = size_t(h) * w * cy;
  for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x) {
    const int ch = int(e % cy), p = int(e / cy), py = p / w, px = p % w;
    if (ch < cx)
      atomicAdd(gx + (size_t(py / 2) * (w / 2) + px / 2) * cx + ch, gy[e]);
    else
      gs[size_t(p) * cs + (ch - cx)] += gy[e];
  }
}

__global__ void k_f32_to_bf16(const float* x, size_t n, __nv_bfloat16* y) {
  for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x)
    y[e] = __float2bfloat16_rn(x[e]);
}

// loss = mean (out - t)^2; g = 2 (out - t) / n
__global__ void k_mse(const float* out, const float* t, int n, float* g, float* loss) {
  __shared__ float sh[32];
  float s = 0.0f;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const float d = out[e] - t[e];
    g[e] = 2.0f * d / float(n);
    s += d * d;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    float r = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0f;
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    if (threadIdx.x == 0) atomicAdd(loss, r / float(n));
  }
}

__global__ void k_adam(float* p, const float* g, float* m, float* v, size_t n, float lr, float b1, float b2, float c1,
                       float c2) {
  for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x) {
    const float gi = g[e];
    const float mi = b1 * m[e] + (1 - b1) * gi, vi = b2 * v[e] + (1 - b2) * gi * gi;
    m[e] = mi;
    v[e] = vi;
    p[e] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
  }
}

// BF16 copy [cout_p][kpad] and transpose [kpad][cout_p] of the FP32 weights [cout][kpad]
__global__ void k_weights(const float* w, int cout, int cout_p, int kpad, __nv_bfloat16* wb, __nv_bfloat16* wt) {
  const size_t n = size_t(cout_p) * kpad;
  for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x) {
    const int o = int(e / kpad), k = int(e % kpad);
    const __nv_bfloat16 v = __float2bfloat16_rn(o < cout ? w[size_t(o) * kpad + k] : 0.0f);
    wb[e] = v;
    wt[size_t(k) * cout_p + o] = v;
  }
}

}  // namespace

WarmStartNet::WarmStartNet(int h, int w, uint64_t seed, cudaStream_t s, int cin0, const int (&c)[4])
    : stream(s), h_(h), w_(w), cin0_(cin0) {
  if (h % 8 || w % 8 || h < 8 || w < 8) throw std::invalid_argument("network grid must be a multiple of 8");
  if (cin0 < 1 || c[0] < 1 || c[1] < 1 || c[2] < 1 || c[3] < 1) throw std::invalid_argument("network widths");
  struct Spec {
    int cin, cout;
    bool relu;
  };
  // encoder: two convolutions per level (widths c0..c3); decoder: one per
  // level on the upsampled coarser output concatenated with the skip
  const Spec specs[12] = {{cin0, c[0], true},        {c[0], c[0], true},        {c[0], c[1], true},
                          {c[1], c[1], true},        {c[1], c[2], true},        {c[2], c[2], true},
                          {c[2], c[3], true},        {c[3], c[3], true},        {c[3] + c[2], c[2], true},
                          {c[2] + c[1], c[1], true}, {c[1] + c[0], c[0], true}, {c[0], 1, false}};
  std::mt19937_64 rng(seed);
  size_t max_col = 0, max_gcol = 0, max_gy = 0;
  const int level_of[12] = {0, 0, 1, 1, 2, 2, 3, 3, 2, 1, 0, 0};
  for (int i = 0; i < 12; ++i) {
    ConvLayer L;
    L.cin = specs[i].cin;
    L.cout = specs[i].cout;
    L.relu = specs[i].relu;
    L.kpad = rup(9 * L.cin, 32);
    L.cout_p = rup(L.cout, 32);
    const size_t nw = size_t(L.cout) * L.kpad;
    std::vector<float> hw(nw, 0.0f), hb(L.cout, 0.0f);
    // He initialisation (the output layer small)
    const float sd = (i == 11 ? 0.1f : 1.0f) * std::sqrt(2.0f / (9.0f * L.cin));
    std::normal_distribution<float> nd(0.0f, sd);
    for (int o = 0; o < L.cout; ++o)
      for (int k = 0; k < 9 * L.cin; ++k) hw[size_t(o) * L.kpad + k] = nd(rng);
    L.w.resize(nw);
    L.b.resize(L.cout);
    GP_CUDA(cudaMemcpy(L.w.get(), hw.data(), nw * 4, cudaMemcpyHostToDevice));
    GP_CUDA(cudaMemcpy(L.b.get(), hb.data(), size_t(L.cout) * 4, cudaMemcpyHostToDevice));
    L.wb.resize(size_t(L.cout_p) * L.kpad);
    L.wt.resize(size_t(L.kpad) * L.cout_p);
    L.gw.resize(nw, true);
    L.gb.resize(L.cout, true);
    L.mw.resize(nw, true);
    L.vw.resize(nw, true);
    L.mb.resize(L.cout, true);
    L.vb.resize(L.cout, true);
    const int lh = h >> level_of[i], lw = w >> level_of[i];
    const size_t rows = size_t(rup(lh * lw, 128));
    max_col = std::max(max_col, rows * L.kpad);
    max_gcol = std::max(max_gcol, rows * L.kpad);
    max_gy = std::max(max_gy, rows * size_t(std::max(L.cout_p, 128)));
    layers_.push_back(std::move(L));
  }
  // activations (see the forward pass for their roles)
  const int chans[19] = {cin0, c[0], c[0], c[0], c[1], c[1], c[1], c[2], c[2], c[2], c[3], c[3], c[3] + c[2],
                         c[2], c[2] + c[1], c[1], c[1] + c[0], c[0], 1};
  const int lev[19] = {0, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 3, 2, 2, 1, 1, 0, 0, 0};
  for (int i = 0; i < 19; ++i) {
    Act a;
    a.h = h >> lev[i];
    a.w = w >> lev[i];
    a.c = chans[i];
    a.y.resize(size_t(a.h) * a.w * a.c, true);
    a.g.resize(size_t(a.h) * a.w * a.c, true);
    acts_.push_back(std::move(a));
  }
  col_.resize(max_col);
  colT_.resize(max_col);
  gcol_.resize(max_gcol);
  gyb_.resize(max_gy);
  gyT_.resize(max_gy);
  out_.resize(size_t(h) * w, true);
  gout_.resize(size_t(h) * w, true);
  loss_.resize(1, true);
  err_.resize(1, true);
  sync_weights();
}

void WarmStartNet::sync_weights() {
  for (auto& L : layers_) {
    k_weights<<<grid_for(size_t(L.cout_p) * L.kpad), kT, 0, stream>>>(L.w.get(), L.cout, L.cout_p, L.kpad, L.wb.get(),
                                                                        L.wt.get());
    GP_LAUNCH_CHECK();
  }
}

double WarmStartNet::flops_forward() const {
  const int level_of[12] = {0, 0, 1, 1, 2, 2, 3, 3, 2, 1, 0, 0};
  double f = 0;
  for (int i = 0; i < 12; ++i) {
    const double hw = double(h_ >> level_of[i]) * double(w_ >> level_of[i]);
    f += 2.0 * hw * 9.0 * layers_[i].cin * layers_[i].cout;
  }
  return f;
}

void WarmStartNet::conv_forward(ConvLayer& L, const Act& x, Act& y, float* out_f32) {
  const int hw = x.h * x.w, rows = rup(hw, 128);
  // implicit im2col inside the GEMM when each K step stays in one tap
  ConvA conv;
  if (L.kpad == 9 * L.cin && L.cin % 32 == 0) {
    conv.x = x.y.get();
    conv.h = x.h;
    conv.w = x.w;
    conv.cin = x.c;
  } else {
    im2col(x, L.kpad, rows);
  }
  GemmEpilogue ep;
  ep.bias = L.b.get();
  ep.relu = L.relu ? 1 : 0;
  ep.ldo = L.cout;
  ep.m_valid = hw;
  ep.n_valid = L.cout;
  if (out_f32)
    ep.out_f32 = out_f32;
  else
    ep.out_bf16 = y.y.get();
  gemm_bf16(col_.get(), L.wb.get(), rows, L.cout_p, L.kpad, ep, err_.get(), stream, conv);
}

void WarmStartNet::im2col(const Act& x, int kpad, int rows) {
  if (x.c % 8 == 0) {
    const size_t chunks = size_t(rows) * (kpad / 8);
    k_im2col8<<<grid_for(chunks), kT, 0, stream>>>(x.y.get(), x.h, x.w, x.c, kpad, rows, col_.get());
  } else {
    k_im2col<<<grid_for(size_t(rows) * kpad), kT, 0, stream>>>(x.y.get(), x.h, x.w, x.c, kpad, rows, col_.get());
  }
  GP_LAUNCH_CHECK();
}

void WarmStartNet::conv_backward(ConvLayer& L, const Act& x, Act& y, Act* dx, const float* gy_override) {
  const int hw = x.h * x.w, rows = rup(hw, 128);
  const float* g = gy_override ? gy_override : y.g.get();
  // pre-activation gradient (BF16, [rows][cout_p]) and the bias gradient
  GP_CUDA(cudaMemsetAsync(L.gb.get(), 0, size_t(L.cout) * 4, stream));
  k_act_back<<<grid_for(size_t(rows) * L.cout_p), kT, 0, stream>>>(g, y.y.get(), hw, L.cout, L.cout_p, rows,
                                                                     L.relu ? 1 : 0, gyb_.get(), L.gb.get());
  GP_LAUNCH_CHECK();
  // weight gradient: gw [cout][kpad] = gy^T [cout_pm x rows] * col^T [kpad x rows]^T
  const int cout_pm = rup(L.cout_p, 128);
  im2col(x, L.kpad, rows);
  {
    dim3 b(32, 8);
    dim3 g1((L.cout_p + 31) / 32, (rows + 31) / 32);
    k_transpose<<<g1, b, 0, stream>>>(gyb_.get(), rows, L.cout_p, L.cout_p, gyT_.get(), cout_pm, rows);
    GP_LAUNCH_CHECK();
    dim3 g2((L.kpad + 31) / 32, (rows + 31) / 32);
    k_transpose<<<g2, b, 0, stream>>>(col_.get(), rows, L.kpad, L.kpad, colT_.get(), L.kpad, rows);
    GP_LAUNCH_CHECK();
  }
  GemmEpilogue ew;
  ew.out_f32 = L.gw.get();
  ew.ldo = L.kpad;
  ew.m_valid = L.cout;
  ew.n_valid = L.kpad;
  ew.split_k = 1;
  gemm_bf16(gyT_.get(), colT_.get(), cout_pm, L.kpad, rows, ew, err_.get(), stream);
  if (!dx) return;
  // input gradient: gcol [rows][kpad] = gy [rows x cout_p] * wt [kpad x cout_p]^T, then col2im
  GemmEpilogue ex;
  ex.out_f32 = gcol_.get();
  ex.ldo = L.kpad;
  ex.m_valid = rows;
  ex.n_valid = L.kpad;
  gemm_bf16(gyb_.get(), L.wt.get(), rows, L.kpad, L.cout_p, ex, err_.get(), stream);
  k_col2im_add<<<grid_for(size_t(hw) * x.c), kT, 0, stream>>>(gcol_.get(), x.h, x.w, x.c, L.kpad, dx->g.get());
  GP_LAUNCH_CHECK();
}

void WarmStartNet::forward(const float* in, float* out) {
  auto& A = acts_;
  const size_t n0 = size_t(h_) * w_ * cin0_;
  k_f32_to_bf16<<<grid_for(n0), kT, 0, stream>>>(in, n0, A[0].y.get());
  GP_LAUNCH_CHECK();
  auto pool = [&](int a, int b) {
    k_pool<<<grid_for(A[b].y.size()), kT, 0, stream>>>(A[a].y.get(), A[a].h, A[a].w, A[a].c, A[b].y.get());
    GP_LAUNCH_CHECK();
  };
  auto up = [&](int x, int sk, int y) {
    k_up_concat<<<grid_for(A[y].y.size()), kT, 0, stream>>>(A[x].y.get(), A[x].c, A[sk].y.get(), A[sk].c, A[y].h,
                                                             A[y].w, A[y].y.get());
    GP_LAUNCH_CHECK();
  };
  conv_forward(layers_[0], A[0], A[1]);
  conv_forward(layers_[1], A[1], A[2]);
  pool(2, 3);
  conv_forward(layers_[2], A[3], A[4]);
  conv_forward(layers_[3], A[4], A[5]);
  pool(5, 6);
  conv_forward(layers_[4], A[6], A[7]);
  conv_forward(layers_[5], A[7], A[8]);
  pool(8, 9);
  conv_forward(layers_[6], A[9], A[10]);
  conv_forward(layers_[7], A[10], A[11]);
  up(11, 8, 12);
  conv_forward(layers_[8], A[12], A[13]);
  up(13, 5, 14);
  conv_forward(layers_[9], A[14], A[15]);
  up(15, 2, 16);
  conv_forward(layers_[10], A[16], A[17]);
  conv_forward(layers_[11], A[17], A[18], out);
}

float WarmStartNet::loss_and_grad(const float* in, const float* target) {
  forward(in, out_.get());
  const int n = h_ * w_;
  GP_CUDA(cudaMemsetAsync(loss_.get(), 0, 4, stream));
  k_mse<<<std::min(grid_for(size_t(n)), 1184), kT, 0, stream>>>(out_.get(), target, n, gout_.get(), loss_.get());
  GP_LAUNCH_CHECK();
  backward(gout_.get());
  float loss = 0;
  int err = 0;
  GP_CUDA(cudaMemcpyAsync(&loss, loss_.get(), 4, cudaMemcpyDeviceToHost, stream));
  GP_CUDA(cudaMemcpyAsync(&err, err_.get(), 4, cudaMemcpyDeviceToHost, stream));
  GP_CUDA(cudaStreamSynchronize(stream));
  if (err) throw std::runtime_error("tensor-core GEMM: MMA completion wait timed out");
  return loss;
}

float WarmStartNet::loss_and_grad_residual(const float* in, const kern::PoissonLayout& L) {
  if (cin0_ != 1) throw std::invalid_argument("the residual loss needs a one-channel network");
  forward(in, out_.get());
  if (!res_.size()) {
    res_.resize(size_t(h_) * w_, true);
    lossd_.resize(1, true);
  }
  GP_CUDA(cudaMemsetAsync(lossd_.get(), 0, sizeof(double), stream));
  residual_loss_grad(out_.get(), in, L, h_, w_, res_.get(), gout_.get(), lossd_.get(), stream);
  backward(gout_.get());
  double loss = 0;
  int err = 0;
  GP_CUDA(cudaMemcpyAsync(&loss, lossd_.get(), sizeof(double), cudaMemcpyDeviceToHost, stream));
  GP_CUDA(cudaMemcpyAsync(&err, err_.get(), 4, cudaMemcpyDeviceToHost, stream));
  GP_CUDA(cudaStreamSynchronize(stream));
  if (err) throw std::runtime_error("tensor-core GEMM: MMA completion wait timed out");
  return float(loss);
}

void WarmStartNet::backward(const float* gout) {
  auto& A = acts_;
  for (auto& a : A) GP_CUDA(cudaMemsetAsync(a.g.get(), 0, a.g.bytes(), stream));
  auto pool_back = [&](int b, int a) {
    k_pool_back<<<grid_for(A[a].g.size()), kT, 0, stream>>>(A[b].g.get(), A[a].h, A[a].w, A[a].c, A[a].g.get());
    GP_LAUNCH_CHECK();
  };
  auto up_back = [&](int y, int x, int sk) {
    k_up_concat_back<<<grid_for(A[y].g.size()), kT, 0, stream>>>(A[y].g.get(), A[x].c, A[sk].c, A[y].h, A[y].w,
                                                                  A[x].g.get(), A[sk].g.get());
    GP_LAUNCH_CHECK();
  };
  conv_backward(layers_[11], A[17], A[18], &A[17], gout);
  conv_backward(layers_[10], A[16], A[17], &A[16]);
  up_back(16, 15, 2);
  conv_backward(layers_[9], A[14], A[15], &A[14]);
  up_back(14, 13, 5);
  conv_backward(layers_[8], A[12], A[13], &A[12]);
  up_back(12, 11, 8);
  conv_backward(layers_[7], A[10], A[11], &A[10]);
  conv_backward(layers_[6], A[9], A[10], &A[9]);
  pool_back(9, 8);
  conv_backward(layers_[5], A[7], A[8], &A[7]);
  conv_backward(layers_[4], A[6], A[7], &A[6]);
  pool_back(6, 5);
  conv_backward(layers_[3], A[4], A[5], &A[4]);
  conv_backward(layers_[2], A[3], A[4], &A[3]);
  pool_back(3, 2);
  conv_backward(layers_[1], A[1], A[2], &A[1]);
  conv_backward(layers_[0], A[0], A[1], nullptr);
}

float WarmStartNet::train_step(const float* in, const float* target, float lr) {
  const float loss = loss_and_grad(in, target);
  adam(lr);
  return loss;
}

float WarmStartNet::train_step_residual(const float* in, const kern::PoissonLayout& L, float lr) {
  const float loss = loss_and_grad_residual(in, L);
  adam(lr);
  return loss;
}

void WarmStartNet::adam(float lr) {
  ++step_;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - std::pow(b1, float(step_)), c2 = 1.0f - std::pow(b2, float(step_));
  for (auto& L : layers_) {
    k_adam<<<grid_for(L.w.size()), kT, 0, stream>>>(L.w.get(), L.gw.get(), L.mw.get(), L.vw.get(), L.w.size(), lr, b1,
                                                    b2, c1, c2);
    GP_LAUNCH_CHECK();
    k_adam<<<grid_for(L.b.size()), kT, 0, stream>>>(L.b.get(), L.gb.get(), L.mb.get(), L.vb.get(), L.b.size(), lr, b1,
                                                    b2, c1, c2);
    GP_LAUNCH_CHECK();
  }
  sync_weights();
}

}  // namespace nn
}  // namespace gample
