// multigrid.cu -- geometric multigrid Poisson solver (sm_100a).
#include "multigrid.hpp"

#include <cfloat>
#include <cmath>
#include <stdexcept>

namespace gample {

namespace {

struct LevelDesc {
  int mx, my;
  int perx, pery;
  float cx, cy, cd;
};

__device__ __forceinline__ float ld(const float* u, const LevelDesc& d, int i, int j) {
  if (i < 0 || i >= d.mx) {
    if (!d.perx) return 0.0f;
    i = (i + d.mx) % d.mx;
  }
  if (j < 0 || j >= d.my) {
    if (!d.pery) return 0.0f;
    j = (j + d.my) % d.my;
  }
  return u[i + j * d.mx];
}

__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (wid == 0) {
    r = lane < int(blockDim.x >> 5) ? sh[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
  }
  __syncthreads();
  return r;
}

// r = b - A x in FP64 with the CSR row of src/EMField.mm:329-400
// (diagonal, i-1, i+1, j-1, j+1); stores float(r) and sum(r), sum(r^2).
__global__ void k_residual64(const double* __restrict__ x, const double* __restrict__ b, kern::PoissonLayout L,
                             float* __restrict__ r32, double* sums) {
  __shared__ double sh[32];
  const int mx = L.nkx + 1, my = L.nky + 1, n = mx * my;
  double s1 = 0.0, s2 = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int i = k % mx, j = k / mx;
    double ax = L.Cd * x[k];
    if (i > 0)
      ax += L.Cx * x[k - 1];
    else if (L.periodic_x)
      ax += L.Cx * x[k + L.nkx];
    if (i < L.nkx)
      ax += L.Cx * x[k + 1];
    else if (L.periodic_x)
      ax += L.Cx * x[k - L.nkx];
    if (j > 0)
      ax += L.Cy * x[k - mx];
    else if (L.periodic_y)
      ax += L.Cy * x[k + L.nky * mx];
    if (j < L.nky)
      ax += L.Cy * x[k + mx];
    else if (L.periodic_y)
      ax += L.Cy * x[k - L.nky * mx];
    const double r = b[k] - ax;
    r32[k] = float(r);
    s1 += r;
    s2 += r * r;
  }
  s1 = block_sum(s1, sh);
  s2 = block_sum(s2, sh);
  if (threadIdx.x == 0) {
    atomicAdd(sums, s1);
    atomicAdd(sums + 1, s2);
  }
}

__global__ void k_sub_mean32(float* f, int n, const double* sums) {
  const float m = float(sums[0] / double(n));
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) f[k] -= m;
}

__global__ void k_axpy(double* x, const float* e, int n) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) x[k] += double(e[k]);
}

__global__ void k_sum64(const double* x, int n, double* sums) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) s += x[k];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) atomicAdd(sums, s);
}

__global__ void k_sub_mean64(double* x, int n, const double* sums) {
  const double m = sums[0] / double(n);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) x[k] -= m;
}

// Red-black Gauss-Seidel half sweep: points with (i + j) % 2 == color.
__global__ void k_smooth(float* __restrict__ u, const float* __restrict__ f, LevelDesc d, int color) {
  const int hx = (d.mx + 1) / 2;
  const int n = hx * d.my;
  const float inv = 1.0f / d.cd;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int j = t / hx;
    const int i = 2 * (t % hx) + ((j + color) & 1);
    if (i >= d.mx) continue;
    const float s = d.cx * (ld(u, d, i - 1, j) + ld(u, d, i + 1, j)) + d.cy * (ld(u, d, i, j - 1) + ld(u, d, i, j + 1));
    u[i + j * d.mx] = (f[i + j * d.mx] - s) * inv;
  }
}

__global__ void k_residual32(const float* __restrict__ u, const float* __restrict__ f, float* __restrict__ r,
                             LevelDesc d) {
  const int n = d.mx * d.my;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int i = k % d.mx, j = k / d.mx;
    const float au = d.cd * u[k] + d.cx * (ld(u, d, i - 1, j) + ld(u, d, i + 1, j)) +
                     d.cy * (ld(u, d, i, j - 1) + ld(u, d, i, j + 1));
    r[k] = f[k] - au;
  }
}

// Full weighting; coarse I sits on fine 2I+1 (Dirichlet) or 2I (periodic).
__global__ void k_restrict(const float* __restrict__ rf, LevelDesc fd, float* __restrict__ fc, LevelDesc cd) {
  const int n = cd.mx * cd.my;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int I = k % cd.mx, J = k / cd.mx;
    const int fi = fd.perx ? 2 * I : 2 * I + 1;
    const int fj = fd.pery ? 2 * J : 2 * J + 1;
    float s = 0.0f;
#pragma unroll
    for (int b = -1; b <= 1; ++b) {
      const float wb = b == 0 ? 0.5f : 0.25f;
#pragma unroll
      for (int a = -1; a <= 1; ++a) {
        const float wa = a == 0 ? 0.5f : 0.25f;
        s += wa * wb * ld(rf, fd, fi + a, fj + b);
      }
    }
    fc[k] = s;
  }
}

// Bilinear interpolation of the coarse correction, added to the fine level.
__device__ __forceinline__ void interp1d(int i, int per, int mc, int& i0, float& w0, int& i1, float& w1) {
  if (per) {
    if ((i & 1) == 0) {
      i0 = i / 2;
      w0 = 1.0f;
      i1 = i0;
      w1 = 0.0f;
    } else {
      i0 = (i - 1) / 2;
      i1 = ((i + 1) / 2) % mc;
      w0 = w1 = 0.5f;
    }
  } else {
    if (i & 1) {
      i0 = (i - 1) / 2;
      w0 = 1.0f;
      i1 = i0;
      w1 = 0.0f;
    } else {
      i0 = i / 2 - 1;
      i1 = i / 2;
      w0 = i0 >= 0 ? 0.5f : 0.0f;
      w1 = i1 < mc ? 0.5f : 0.0f;
      if (i0 < 0) i0 = 0;
      if (i1 >= mc) i1 = mc - 1;
    }
  }
}

__global__ void k_prolong(const float* __restrict__ uc, LevelDesc cd, float* __restrict__ uf, LevelDesc fd) {
  const int n = fd.mx * fd.my;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int i = k % fd.mx, j = k / fd.mx;
    int a0, a1, b0, b1;
    float wa0, wa1, wb0, wb1;
    interp1d(i, fd.perx, cd.mx, a0, wa0, a1, wa1);
    interp1d(j, fd.pery, cd.my, b0, wb0, b1, wb1);
    const float e = wb0 * (wa0 * uc[a0 + b0 * cd.mx] + wa1 * uc[a1 + b0 * cd.mx]) +
                    wb1 * (wa0 * uc[a0 + b1 * cd.mx] + wa1 * uc[a1 + b1 * cd.mx]);
    uf[k] += e;
  }
}

// Coarsest level: CG on (-A) u = -f in one block; work holds 3 vectors.
__global__ void __launch_bounds__(1024) k_coarse_cg(float* u, const float* f, LevelDesc d, float* work, int maxit,
                                                    float rtol) {
  __shared__ double sh[32];
  __shared__ double s_val;
  const int n = d.mx * d.my;
  float* r = work;
  float* p = work + n;
  float* q = work + 2 * n;
  const bool singular = d.perx && d.pery;
  double mean = 0.0;
  if (singular) {
    double s = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) s += f[k];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) s_val = s / n;
    __syncthreads();
    mean = s_val;
  }
  double rr = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const float v = -(f[k] - float(mean));
    u[k] = 0.0f;
    r[k] = v;
    p[k] = v;
    rr += double(v) * v;
  }
  rr = block_sum(rr, sh);
  if (threadIdx.x == 0) s_val = rr;
  __syncthreads();
  rr = s_val;
  const double stop = double(rtol) * double(rtol) * rr;
  for (int it = 0; it < maxit && rr > stop && rr > 0.0; ++it) {
    double pq = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      const int i = k % d.mx, j = k / d.mx;
      const float ap = d.cd * p[k] + d.cx * (ld(p, d, i - 1, j) + ld(p, d, i + 1, j)) +
                       d.cy * (ld(p, d, i, j - 1) + ld(p, d, i, j + 1));
      q[k] = -ap;
      pq += double(p[k]) * double(-ap);
    }
    pq = block_sum(pq, sh);
    if (threadIdx.x == 0) s_val = pq;
    __syncthreads();
    pq = s_val;
    if (!(pq > 0.0)) break;
    const float alpha = float(rr / pq);
    double rn = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      u[k] += alpha * p[k];
      r[k] -= alpha * q[k];
      rn += double(r[k]) * r[k];
    }
    rn = block_sum(rn, sh);
    if (threadIdx.x == 0) s_val = rn;
    __syncthreads();
    rn = s_val;
    const float beta = float(rn / rr);
    rr = rn;
    for (int k = threadIdx.x; k < n; k += blockDim.x) p[k] = r[k] + beta * p[k];
    __syncthreads();
  }
  if (singular) {
    double s = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) s += u[k];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) s_val = s / n;
    __syncthreads();
    const float m = float(s_val);
    for (int k = threadIdx.x; k < n; k += blockDim.x) u[k] -= m;
  }
}

int blocks_for(int n, int per_thread = 1) {
  long long b = ((long long)n + 256LL * per_thread - 1) / (256LL * per_thread);
  if (b < 1) b = 1;
  return int(b < 2368 ? b : 2368);
}

LevelDesc desc(const PoissonMG::Level& l) { return LevelDesc{l.mx, l.my, l.perx, l.pery, l.cx, l.cy, l.cd}; }

bool can_coarsen(int n, bool per) { return per ? (n >= 4 && n % 2 == 0) : (n >= 3 && n % 2 == 1); }

}  // namespace

PoissonMG::PoissonMG(const kern::PoissonLayout& L, int nu_pre, int nu_post)
    : L_(L), nu_pre_(nu_pre), nu_post_(nu_post), sums_(2, true), host_(4) {
  if (!((L.fbc[0] == kern::FBC_PERIODIC_C) == (L.fbc[1] == kern::FBC_PERIODIC_C)) ||
      !((L.fbc[2] == kern::FBC_PERIODIC_C) == (L.fbc[3] == kern::FBC_PERIODIC_C)))
    throw std::invalid_argument("periodic field boundaries must be set on both walls of a direction");
  for (int w = 0; w < 4; ++w)
    if (L.fbc[w] != kern::FBC_PERIODIC_C && L.fbc[w] != kern::FBC_DIRICHLET_C)
      throw std::invalid_argument("field boundary must be Dirichlet or periodic (Neumann is rejected as in "
                                  "the reference's Poisson set-up)");
  int mx = L.nkx + 1, my = L.nky + 1;
  if (mx < 1 || my < 1) throw std::invalid_argument("empty Poisson system");
  n_ = mx * my;
  float cx = float(L.Cx), cy = float(L.Cy);
  for (;;) {
    Level lv;
    lv.mx = mx;
    lv.my = my;
    lv.perx = L.periodic_x;
    lv.pery = L.periodic_y;
    lv.cx = cx;
    lv.cy = cy;
    lv.cd = -2.0f * (cx + cy);
    lv.u.resize(size_t(mx) * my, true);
    lv.f.resize(size_t(mx) * my, true);
    lv.r.resize(size_t(mx) * my, true);
    lv_.push_back(std::move(lv));
    if (!(can_coarsen(mx, L.periodic_x) && can_coarsen(my, L.periodic_y))) break;
    if (size_t(mx) * my <= 16) break;
    mx = L.periodic_x ? mx / 2 : (mx - 1) / 2;
    my = L.periodic_y ? my / 2 : (my - 1) / 2;
    cx *= 0.25f;
    cy *= 0.25f;
  }
  const Level& c = lv_.back();
  cg_work_.resize(3 * size_t(c.mx) * c.my, true);
}

void PoissonMG::vcycle_level(int l, cudaStream_t s) {
  Level& a = lv_[l];
  const LevelDesc d = desc(a);
  const int n = a.mx * a.my;
  if (l + 1 == int(lv_.size())) {
    const int maxit = n * 2 + 10 < 2000 ? n * 2 + 10 : 2000;
    k_coarse_cg<<<1, 1024, 0, s>>>(a.u.get(), a.f.get(), d, cg_work_.get(), maxit, 1e-5f);
    GP_LAUNCH_CHECK();
    return;
  }
  Level& b = lv_[l + 1];
  const int hb = blocks_for((a.mx + 1) / 2 * a.my);
  GP_CUDA(cudaMemsetAsync(a.u.get(), 0, size_t(n) * sizeof(float), s));
  for (int it = 0; it < nu_pre_; ++it) {
    k_smooth<<<hb, 256, 0, s>>>(a.u.get(), a.f.get(), d, 0);
    GP_LAUNCH_CHECK();
    k_smooth<<<hb, 256, 0, s>>>(a.u.get(), a.f.get(), d, 1);
    GP_LAUNCH_CHECK();
  }
  k_residual32<<<blocks_for(n), 256, 0, s>>>(a.u.get(), a.f.get(), a.r.get(), d);
  GP_LAUNCH_CHECK();
  k_restrict<<<blocks_for(b.mx * b.my), 256, 0, s>>>(a.r.get(), d, b.f.get(), desc(b));
  GP_LAUNCH_CHECK();
  vcycle_level(l + 1, s);
  k_prolong<<<blocks_for(n), 256, 0, s>>>(b.u.get(), desc(b), a.u.get(), d);
  GP_LAUNCH_CHECK();
  for (int it = 0; it < nu_post_; ++it) {
    k_smooth<<<hb, 256, 0, s>>>(a.u.get(), a.f.get(), d, 1);
    GP_LAUNCH_CHECK();
    k_smooth<<<hb, 256, 0, s>>>(a.u.get(), a.f.get(), d, 0);
    GP_LAUNCH_CHECK();
  }
}

void PoissonMG::vcycle(cudaStream_t s) { vcycle_level(0, s); }

MGResult PoissonMG::solve(const double* b, const double* sums_b, double* x, double tol, int maxiter,
                          cudaStream_t s) {
  MGResult res;
  GP_CUDA(cudaMemcpyAsync(host_.get(), sums_b, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  GP_CUDA(cudaStreamSynchronize(s));
  res.norm_b = std::sqrt(host_[1] > 0 ? host_[1] : 0.0);
  if (res.norm_b < DBL_EPSILON) {  // AMGCL clears x for a zero right-hand side
    GP_CUDA(cudaMemsetAsync(x, 0, size_t(n_) * sizeof(double), s));
    res.rel_residual = res.norm_b;
    return res;
  }
  Level& f = lv_[0];
  const bool singular = L_.periodic_x && L_.periodic_y;
  for (int it = 0;; ++it) {
    GP_CUDA(cudaMemsetAsync(sums_.get(), 0, 2 * sizeof(double), s));
    k_residual64<<<blocks_for(n_), 256, 0, s>>>(x, b, L_, f.f.get(), sums_.get());
    GP_LAUNCH_CHECK();
    GP_CUDA(cudaMemcpyAsync(host_.get(), sums_.get(), 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    GP_CUDA(cudaStreamSynchronize(s));
    res.rel_residual = std::sqrt(host_[1] > 0 ? host_[1] : 0.0) / res.norm_b;
    res.iterations = it;
    if (!(res.rel_residual > tol) || it >= maxiter) break;
    if (singular) {
      k_sub_mean32<<<blocks_for(n_), 256, 0, s>>>(f.f.get(), n_, sums_.get());
      GP_LAUNCH_CHECK();
    }
    vcycle_level(0, s);
    k_axpy<<<blocks_for(n_), 256, 0, s>>>(x, f.u.get(), n_);
    GP_LAUNCH_CHECK();
  }
  if (singular) {
    GP_CUDA(cudaMemsetAsync(sums_.get(), 0, sizeof(double), s));
    k_sum64<<<blocks_for(n_), 256, 0, s>>>(x, n_, sums_.get());
    GP_LAUNCH_CHECK();
    k_sub_mean64<<<blocks_for(n_), 256, 0, s>>>(x, n_, sums_.get());
    GP_LAUNCH_CHECK();
  }
  return res;
}

}  // namespace gample
