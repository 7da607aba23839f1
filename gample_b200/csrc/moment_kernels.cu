// moment_kernels.cu -- velocity moments of one species (sm_100a).
//
// Restates the integrateMoments kernel (src/Moment.mm:33-135) and the host
// normalisation (src/Moment.mm:287-316). Per node, with the node-centred
// B-spline weights s of each particle at its reference position
// x = ix + ox (cell from int(x), as src/Moment.mm:67-68 truncates):
//   n += s * scale,  u_a += s * v_a,  P_ab += s * v_a * v_b
// then u_a /= n / scale and P_ab = m (P_ab / (n / scale) - u_a u_b) n.
//
// One CTA per chunk of 2048 consecutive (cell-sorted) particles: the ten
// sums of the chunk's box are accumulated in shared memory (FP32, each lane
// visiting the stencil in its own rotated order so that lanes sharing a cell
// rarely collide) and flushed with one FP64 global atomic per node and
// quantity; particles outside the box add to global memory directly.
#include <cuda_runtime.h>

#include <climits>
#include <stdexcept>

#include "device.hpp"
#include "kernels.hpp"
#include "pic_common.cuh"

namespace gample {
namespace kern {

namespace {

constexpr int kThreads = 256;
constexpr int kPer = 8;
constexpr int kChunk = kThreads * kPer;
constexpr int kWin = 1152;   // window entries per quantity (ten fit the 48 KB of static shared memory)
constexpr int kReach = 12;   // box: cells within kReach of the chunk's middle particle
constexpr int kQ = 10;       // n, ux, uy, uz, Pxx, Pxy, Pxz, Pyy, Pyz, Pzz

struct Box {
  int use, x0, y0, w, h;  // window origin (node indices) and size
};

// r[t] = w[(t + sh) mod N] for a per-lane shift sh in [0, N).
template <int N>
__device__ __forceinline__ void rotated(const float (&w)[N], int sh, float (&r)[N]) {
#pragma unroll
  for (int t = 0; t < N; ++t) {
    float v = w[t];
#pragma unroll
    for (int q = 1; q < N; ++q)
      if (sh == q) v = w[(t + q) % N];
    r[t] = v;
  }
}

// Reference position of a particle and its truncated cell (src/Moment.mm:67-71).
__device__ __forceinline__ void ref_cell(int32_t cell, float ox, float oy, int& i1, int& j1, float& hx, float& hy) {
  const float x = __fadd_rn(float(cell_ix(cell)), ox), y = __fadd_rn(float(cell_iy(cell)), oy);
  i1 = int(x);
  j1 = int(y);
  hx = __fsub_rn(x, float(i1));
  hy = __fsub_rn(y, float(j1));
}

template <int ORDER>
__global__ void __launch_bounds__(kThreads) k_moments(GridDims g, ParticleArrays p, const SpeciesCounters* cnt,
                                                      float scale, double* acc, size_t nrho) {
  constexpr int N = ORDER + 1;
  __shared__ float sw[kQ * kWin];
  __shared__ int s_red[4][kThreads / 32];
  __shared__ Box s_box;
  __shared__ int s_ref;
  const uint32_t n = cnt->n;
  const uint32_t base = blockIdx.x * uint32_t(kChunk);
  if (base >= n) return;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int nx = g.nx, ny = g.ny, ngb = g.ngb;

  if (tid == 0) {
    const uint32_t rest = n - base;
    const uint32_t k = base + (rest < uint32_t(kChunk) ? rest / 2 : uint32_t(kChunk / 2));
    const int32_t c = p.cell[k];
    int ri = -1;
    if (c >= 0) {
      int i1, j1;
      float hx, hy;
      ref_cell(c, p.ox[k], p.oy[k], i1, j1, hx, hy);
      ri = i1 | (j1 << 16);
    }
    s_ref = ri;
  }
  __syncthreads();
  const int ref = s_ref;
  const int rx = ref >= 0 ? (ref & 0xFFFF) : 0, ry = ref >= 0 ? (ref >> 16) : 0;
  int mnx = INT_MAX, mny = INT_MAX, mxx = INT_MIN, mxy = INT_MIN;
  for (int i = 0; i < kPer; ++i) {
    const uint32_t k = base + uint32_t(i * kThreads + tid);
    if (k >= n || ref < 0) continue;
    const int32_t c = p.cell[k];
    if (c < 0) continue;
    int i1, j1;
    float hx, hy;
    ref_cell(c, p.ox[k], p.oy[k], i1, j1, hx, hy);
    if (abs(i1 - rx) > kReach || abs(j1 - ry) > kReach) continue;
    mnx = min(mnx, i1);
    mxx = max(mxx, i1);
    mny = min(mny, j1);
    mxy = max(mxy, j1);
  }
  mnx = __reduce_min_sync(0xffffffffu, mnx);
  mny = __reduce_min_sync(0xffffffffu, mny);
  mxx = __reduce_max_sync(0xffffffffu, mxx);
  mxy = __reduce_max_sync(0xffffffffu, mxy);
  if (lane == 0) {
    s_red[0][wid] = mnx;
    s_red[1][wid] = mny;
    s_red[2][wid] = mxx;
    s_red[3][wid] = mxy;
  }
  __syncthreads();
  if (tid == 0) {
    Box b{};
    int a0 = INT_MAX, a1 = INT_MAX, a2 = INT_MIN, a3 = INT_MIN;
    for (int q = 0; q < kThreads / 32; ++q) {
      a0 = min(a0, s_red[0][q]);
      a1 = min(a1, s_red[1][q]);
      a2 = max(a2, s_red[2][q]);
      a3 = max(a3, s_red[3][q]);
    }
    if (a0 != INT_MAX) {
      b.x0 = a0 - ngb;
      b.y0 = a1 - ngb;
      b.w = a2 - a0 + N;
      b.h = a3 - a1 + N;
      b.use = b.w * b.h <= kWin ? 1 : 0;
    }
    s_box = b;
  }
  __syncthreads();
  const Box b = s_box;
  if (b.use)
    for (int e = tid; e < kQ * b.w * b.h; e += kThreads) sw[(e / (b.w * b.h)) * kWin + e % (b.w * b.h)] = 0.0f;
  __syncthreads();

  const int si = lane % N, sj = (lane / N) % N;
  for (int it = 0; it < kPer; ++it) {
    const uint32_t k = base + uint32_t(it * kThreads + tid);
    if (k >= n) continue;
    const int32_t c = p.cell[k];
    if (c < 0) continue;
    int i1, j1;
    float hx, hy;
    ref_cell(c, p.ox[k], p.oy[k], i1, j1, hx, hy);
    float w0x[N], w0y[N], wx[N], wy[N];
    shape<ORDER>(hx, w0x);
    shape<ORDER>(hy, w0y);
    const float vx = p.vx[k], vy = p.vy[k], vz = p.vz[k];
    const bool win = b.use && i1 - ngb >= b.x0 && j1 - ngb >= b.y0 && i1 - ngb + N <= b.x0 + b.w &&
                     j1 - ngb + N <= b.y0 + b.h;
    const int ri = win ? si : 0, rj = win ? sj : 0;
    rotated<N>(w0x, ri, wx);
    rotated<N>(w0y, rj, wy);
#pragma unroll
    for (int a = 0; a < N; ++a)
#pragma unroll
      for (int q = 0; q < N; ++q) {
        const int i = q + ri >= N ? q + ri - N : q + ri, j = a + rj >= N ? a + rj - N : a + rj;
        const float s = __fmul_rn(wx[q], wy[a]);
        const float v[kQ] = {__fmul_rn(s, scale),
                             __fmul_rn(s, vx),
                             __fmul_rn(s, vy),
                             __fmul_rn(s, vz),
                             __fmul_rn(__fmul_rn(s, vx), vx),
                             __fmul_rn(__fmul_rn(s, vx), vy),
                             __fmul_rn(__fmul_rn(s, vx), vz),
                             __fmul_rn(__fmul_rn(s, vy), vy),
                             __fmul_rn(__fmul_rn(s, vy), vz),
                             __fmul_rn(__fmul_rn(s, vz), vz)};
        const int ii = i1 + i - ngb, jj = j1 + j - ngb;
        if (win) {
          const int o = (ii - b.x0) + (jj - b.y0) * b.w;
#pragma unroll
          for (int t = 0; t < kQ; ++t) atomicAdd(sw + t * kWin + o, v[t]);
        } else if (ii >= 0 && jj >= 0 && ii <= nx && jj <= ny) {
          const size_t o = size_t(ii) + size_t(jj) * (nx + 1);
#pragma unroll
          for (int t = 0; t < kQ; ++t) atomicAdd(acc + t * nrho + o, double(v[t]));
        }
      }
  }
  __syncthreads();
  if (b.use)
    for (int e = tid; e < b.w * b.h; e += kThreads) {
      const int ii = b.x0 + e % b.w, jj = b.y0 + e / b.w;
      if (ii < 0 || jj < 0 || ii > nx || jj > ny) continue;
      const size_t o = size_t(ii) + size_t(jj) * (nx + 1);
#pragma unroll
      for (int t = 0; t < kQ; ++t) {
        const float v = sw[t * kWin + e];
        if (v != 0.0f) atomicAdd(acc + t * nrho + o, double(v));
      }
    }
}

// Sums -> moments (src/Moment.mm:287-316), in FP32 with explicit rounding.
__global__ void k_moments_finish(const double* acc, size_t nrho, float scale, float m, float* out) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < nrho; i += size_t(gridDim.x) * blockDim.x) {
    float q[kQ];
#pragma unroll
    for (int t = 0; t < kQ; ++t) q[t] = __double2float_rn(acc[t * nrho + i]);
    const float nn = q[0];
    if (nn > 1e-20f) {
      const float d = __fdiv_rn(nn, scale);
      const float ux = __fdiv_rn(q[1], d), uy = __fdiv_rn(q[2], d), uz = __fdiv_rn(q[3], d);
      const float u[3] = {ux, uy, uz};
      out[1 * nrho + i] = ux;
      out[2 * nrho + i] = uy;
      out[3 * nrho + i] = uz;
      const int pa[6] = {0, 0, 0, 1, 1, 2}, pb[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
      for (int t = 0; t < 6; ++t)
        out[(4 + t) * nrho + i] =
            __fmul_rn(__fmul_rn(m, __fsub_rn(__fdiv_rn(q[4 + t], d), __fmul_rn(u[pa[t]], u[pb[t]]))), nn);
    } else {
#pragma unroll
      for (int t = 1; t < kQ; ++t) out[t * nrho + i] = 0.0f;
    }
    out[i] = nn;
  }
}

int grid1(size_t n) {
  const size_t b = (n + 255) / 256;
  return int(b < 148 * 8 ? (b ? b : 1) : 148 * 8);
}

}  // namespace

void moments(int order, GridDims g, ParticleArrays p, const SpeciesCounters* cnt, uint32_t n_bound, float scale,
             float mass, double* acc, float* out, cudaStream_t s) {
  const size_t nrho = size_t(g.nx + 1) * (g.ny + 1);
  GP_CUDA(cudaMemsetAsync(acc, 0, 10 * nrho * sizeof(double), s));
  if (n_bound) {
    const uint32_t nb = (n_bound + kChunk - 1) / kChunk;
    switch (order) {
      case 1: k_moments<1><<<nb, kThreads, 0, s>>>(g, p, cnt, scale, acc, nrho); break;
      case 3: k_moments<3><<<nb, kThreads, 0, s>>>(g, p, cnt, scale, acc, nrho); break;
      case 5: k_moments<5><<<nb, kThreads, 0, s>>>(g, p, cnt, scale, acc, nrho); break;
      default: throw std::invalid_argument("WeightingOrder must be 1, 3 or 5");
    }
    GP_LAUNCH_CHECK();
  }
  k_moments_finish<<<grid1(nrho), 256, 0, s>>>(acc, nrho, scale, mass, out);
  GP_LAUNCH_CHECK();
}

}  // namespace kern
}  // namespace gample
