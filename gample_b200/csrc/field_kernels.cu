// field_kernels.cu -- grid kernels around the Poisson solve (sm_100a).
//
// All arrays keep the reference's staggered extents and strides
// (src/EMField.mm:127-144). Every kernel here is HBM/launch bound on small
// arrays (about 1 MB per field at 512^2).
#include <cuda_runtime.h>

#include "device.hpp"
#include "pdl.cuh"
#include "kernels.hpp"

namespace gample {
namespace kern {

namespace {

constexpr double kPI = 3.141592653589793;

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
  return r;  // valid in thread 0
}

__global__ void k_fill_f32(float* p, size_t n, float v) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    p[i] = v;
}
__global__ void k_fill_f64(double* p, size_t n, double v) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    p[i] = v;
}

struct AccList {
  const long long* p[4];
  double f[4];
};
struct AccListD {
  const double* p[4];
};

__global__ void k_combine_f64(AccListD a, int ns, size_t n, float* out) {
  grid_dependency_wait();
  grid_dependents_launch();
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    double v = 0.0;
    for (int s = 0; s < ns; ++s) v = __dadd_rn(v, a.p[s][i]);
    out[i] = __double2float_rn(v);
  }
}

__global__ void k_combine(AccList a, int ns, size_t n, float* out) {
  grid_dependency_wait();
  grid_dependents_launch();
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    double v = 0.0;
    for (int s = 0; s < ns; ++s) v = __dadd_rn(v, __dmul_rn(double(a.p[s][i]), a.f[s]));
    out[i] = __double2float_rn(v);
  }
}

// Phase 0: non-periodic x walls, one thread per row j (src/EMField.mm:751-782).
// Phase 1: non-periodic y walls, one thread per column i (:783-814).
// Phase 2: periodic x, per row (:817-832). Phase 3: periodic y, per column (:833-850).
__global__ void k_fold(float* rho, GridDims g, int f0, int f1, int f2, int f3, int phase) {
  grid_dependency_wait();
  grid_dependents_launch();
  const int nx = g.nx, ny = g.ny, ngb = g.ngb, ngx = g.ngx, ngy = g.ngy;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (phase == 0) {
    const int j = t;
    if (j > ny) return;
    float* r = rho + j * (nx + 1);
    if (f0 == FBC_DIRICHLET_C)
      for (int i = 0; i <= ngb; i++) r[ngb + 1] += r[i];
    else if (f0 == FBC_NEUMANN_C)
      for (int i = 0; i < ngb; i++) r[ngb] += r[i];
    if (f1 == FBC_DIRICHLET_C)
      for (int i = 0; i <= ngb; i++) r[ngb + ngx - 1] += r[ngb + ngx + i];
    else if (f1 == FBC_NEUMANN_C)
      for (int i = 0; i < ngb; i++) r[ngb + ngx] += r[ngb + ngx + i];
  } else if (phase == 1) {
    const int i = t;
    if (i > nx) return;
    const int s = nx + 1;
    if (f2 == FBC_DIRICHLET_C)
      for (int j = 0; j <= ngb; j++) rho[i + (ngb + 1) * s] += rho[i + j * s];
    else if (f2 == FBC_NEUMANN_C)
      for (int j = 0; j < ngb; j++) rho[i + ngb * s] += rho[i + j * s];
    if (f3 == FBC_DIRICHLET_C)
      for (int j = 0; j <= ngb; j++) rho[i + (ngb + ngy - 1) * s] += rho[i + (ngb + ngy + j) * s];
    else if (f3 == FBC_NEUMANN_C)
      for (int j = 0; j < ngb; j++) rho[i + (ngb + ngy) * s] += rho[i + (ngb + ngy + j) * s];
  } else if (phase == 2) {
    const int j = t;
    if (j > ny) return;
    float* r = rho + j * (nx + 1);
    for (int i = 0; i < ngb; i++) r[ngx + i] += r[i];
    for (int i = 0; i <= ngb; i++) r[ngb + i] += r[ngb + ngx + i];
  } else {
    const int i = t;
    if (i > nx) return;
    const int s = nx + 1;
    for (int j = 0; j < ngb; j++) rho[i + (ngy + j) * s] += rho[i + j * s];
    for (int j = 0; j <= ngb; j++) rho[i + (ngb + j) * s] += rho[i + (ngb + ngy + j) * s];
  }
}

__global__ void k_rhs(const float* rho, GridDims g, PoissonLayout L, double* b, double* sums) {
  grid_dependency_wait();
  grid_dependents_launch();
  __shared__ double sh[32];
  const int nkx1 = L.nkx + 1, n = nkx1 * (L.nky + 1);
  double s1 = 0.0, s2 = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int i = k % nkx1, j = k / nkx1;
    // _rhs_BC[k] accumulated in the reference's order (src/EMField.mm:333-400)
    double bc = 0.0;
    if (i == 0 && L.fbc[0] == FBC_DIRICHLET_C) bc += -L.Cx * L.phiXmin;
    if (i == L.nkx && L.fbc[1] == FBC_DIRICHLET_C) bc += -L.Cx * L.phiXmax;
    if (j == 0 && L.fbc[2] == FBC_DIRICHLET_C) bc += -L.Cy * L.phiYmin;
    if (j == L.nky && L.fbc[3] == FBC_DIRICHLET_C) bc += -L.Cy * L.phiYmax;
    const double v = __dsub_rn(bc, __dmul_rn(4 * kPI, double(rho[(i + L.ikmin) + (j + L.jkmin) * (g.nx + 1)])));
    b[k] = v;
    s1 += v;
    s2 += v * v;
  }
  s1 = block_sum(s1, sh);
  s2 = block_sum(s2, sh);
  if (threadIdx.x == 0) {
    atomicAdd(sums, s1);
    atomicAdd(sums + 1, s2);
  }
}

__global__ void k_vec_sums(const double* v, int n, double* sums) {
  __shared__ double sh[32];
  double s1 = 0.0, s2 = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    s1 += v[k];
    s2 += v[k] * v[k];
  }
  s1 = block_sum(s1, sh);
  s2 = block_sum(s2, sh);
  if (threadIdx.x == 0) {
    atomicAdd(sums, s1);
    atomicAdd(sums + 1, s2);
  }
}

__global__ void k_subtract_mean(double* v, int n, const double* sum) {
  const double m = sum[0] / double(n);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) v[k] -= m;
}

// Hollow-cathode mean of the solution column (src/EMField.mm:1064-1070).
__global__ void k_cathode_mean(const double* sol, PoissonLayout L, int col, double* out) {
  grid_dependency_wait();
  grid_dependents_launch();
  __shared__ double sh[32];
  double s = 0.0;
  for (int j = threadIdx.x; j <= L.nky; j += blockDim.x) s += sol[col + j * (L.nkx + 1)];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) *out = s / (L.nky + 1);
}

// phi fill (src/EMField.mm:873-1061) + hollow-cathode shift (:1071-1076).
__global__ void k_phi_fill(const double* sol, GridDims g, PoissonLayout L, float dx, double cathode_pos,
                           const double* cathode_mean, double* phi) {
  grid_dependency_wait();
  grid_dependents_launch();
  const int nx = g.nx, ny = g.ny, ngb = g.ngb, ngx = g.ngx, ngy = g.ngy;
  const int nkx = L.nkx, nky = L.nky;
  const int W = nx + 3, H = ny + 3;
  const int* fbc = L.fbc;
  auto S = [&](int i, int j) { return sol[i + j * (nkx + 1)]; };
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < W * H; k += gridDim.x * blockDim.x) {
    const int i = k % W, j = k / W;
    bool isLeft = false, isRight = false, isBottom = false, isTop = false;
    int iin = 0, jin = 0;
    if (fbc[2] == FBC_DIRICHLET_C) {
      isBottom = (j <= ngb + 1);
      jin = j - (ngb + 1) - 1;
    } else if (fbc[2] == FBC_NEUMANN_C) {
      isBottom = (j < ngb + 1);
      jin = j - (ngb + 1);
    } else if (fbc[2] == FBC_PERIODIC_C) {
      jin = ((j - (ngb + 1) + ngy) % ngy + ngy) % ngy;
    }
    if (fbc[3] == FBC_DIRICHLET_C)
      isTop = (j >= ngb + 1 + ngy);
    else if (fbc[3] == FBC_NEUMANN_C)
      isTop = (j > ngb + 1 + ngy);
    if (fbc[0] == FBC_DIRICHLET_C) {
      isLeft = (i <= ngb + 1);
      iin = i - (ngb + 1) - 1;
    } else if (fbc[0] == FBC_NEUMANN_C) {
      isLeft = (i < ngb + 1);
      iin = i - (ngb + 1);
    } else if (fbc[0] == FBC_PERIODIC_C) {
      // +ngx: the reference's "+ngx-1" (src/EMField.mm:907) shifts phi by one
      // cell in x; corrected here (its y branch, :886, uses +ngy).
      iin = ((i - (ngb + 1) + ngx) % ngx + ngx) % ngx;
    }
    if (fbc[1] == FBC_DIRICHLET_C)
      isRight = (i >= ngb + 1 + ngx);
    else if (fbc[1] == FBC_NEUMANN_C)
      isRight = (i > ngb + 1 + ngx);
    double out = 0.0;
    if (!isLeft && !isRight && !isBottom && !isTop) {
      out = S(iin, jin);
    } else if (isLeft != isRight && !isBottom && !isTop) {
      if (isLeft)
        out = L.phiXmin + (i - (ngb + 1)) * (S(0, jin) - L.phiXmin);
      else
        out = L.phiXmax + (i - (ngb + 1 + ngx)) * (L.phiXmax - S(nkx, jin));
    } else if (!isLeft && !isRight && isBottom != isTop) {
      if (isBottom)
        out = L.phiYmin + (j - (ngb + 1)) * (S(iin, 0) - L.phiYmin);
      else
        out = L.phiYmax + (j - (ngb + 1 + ngy)) * (L.phiYmax - S(iin, nky));
    } else if ((isLeft != isRight) && (isBottom != isTop)) {
      // corners with Dirichlet on both walls (Neumann is rejected at set-up)
      const int ci = isLeft ? 0 : nkx, cj = isBottom ? 0 : nky;
      const int ni = isLeft ? 1 : nkx - 1, nj = isBottom ? 1 : nky - 1;
      const double ddx = isLeft ? (S(ni, cj) - S(ci, cj)) : (S(ci, cj) - S(ni, cj));
      const double ddy = isBottom ? (S(ci, nj) - S(ci, cj)) : (S(ci, cj) - S(ci, nj));
      const int di = isLeft ? (i - (ngb + 1)) : (i - (ngb + 1 + ngx));
      const int dj = isBottom ? (j - (ngb + 1)) : (j - (ngb + 1 + ngy));
      out = (isLeft ? L.phiXmin : L.phiXmax) + di * ddx + dj * ddy;
    }
    // (i - ngb - 2) * _dx is an int x float product in the reference.
    if (cathode_pos > 0.0) out -= *cathode_mean * double(__fmul_rn(float(i - ngb - 2), dx)) / cathode_pos;
    phi[k] = out;
  }
}

__global__ void k_gradient(const double* phi, GridDims g, float dx, float dy, float* Ex, float* Ey, const float* jx,
                           const float* jy, double* sums, float* Exp, float* Eyp, int pitch) {
  grid_dependency_wait();
  grid_dependents_launch();
  __shared__ double sh[32];
  const int nx = g.nx, ny = g.ny;
  const int nEx = (nx + 2) * (ny + 1), nEy = (nx + 1) * (ny + 2);
  double e2 = 0.0, ej = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nEx + nEy; k += gridDim.x * blockDim.x) {
    if (k < nEx) {
      const int i = k % (nx + 2), j = k / (nx + 2);
      const double d = phi[i + 1 + (j + 1) * (nx + 3)] - phi[i + (j + 1) * (nx + 3)];
      const float v = __double2float_rn(-d / double(dx));
      Ex[k] = v;
      if (Exp) Exp[i + j * pitch] = v;
      e2 += double(v) * double(v);
      ej += double(v) * double(jx[k]);
    } else {
      const int kk = k - nEx;
      const int i = kk % (nx + 1), j = kk / (nx + 1);
      const double d = phi[i + 1 + (j + 1) * (nx + 3)] - phi[i + 1 + j * (nx + 3)];
      const float v = __double2float_rn(-d / double(dy));
      Ey[kk] = v;
      if (Eyp) Eyp[i + j * pitch] = v;
      e2 += double(v) * double(v);
      ej += double(v) * double(jy[kk]);
    }
  }
  e2 = block_sum(e2, sh);
  ej = block_sum(ej, sh);
  if (threadIdx.x == 0) {
    atomicAdd(sums, e2);
    atomicAdd(sums + 1, ej);
  }
}

__global__ void k_probe(const double* phi, const float* Ex, const float* Ey, GridDims g, double* out) {
  grid_dependency_wait();
  grid_dependents_launch();
  const int p_i = g.ngx / 4 + g.ngb, p_j = g.ngy / 2 + g.ngb, nx = g.nx;
  out[0] = phi[(p_i + 2) + (p_j + 2) * (nx + 3)];
  out[1] = double(Ex[(p_i + 1) + p_j * (nx + 2)]);
  out[2] = double(Ey[p_i + (p_j + 1) * (nx + 1)]);
}

int grid1d(size_t n, int block = 256, int cap = 1184) {
  size_t b = (n + block - 1) / block;
  if (b < 1) b = 1;
  return int(b < size_t(cap) ? b : size_t(cap));
}

}  // namespace

void fill_f32(float* p, size_t n, float v, cudaStream_t s) {
  if (!n) return;
  k_fill_f32<<<grid1d(n), 256, 0, s>>>(p, n, v);
  GP_LAUNCH_CHECK();
}
void fill_f64(double* p, size_t n, double v, cudaStream_t s) {
  if (!n) return;
  k_fill_f64<<<grid1d(n), 256, 0, s>>>(p, n, v);
  GP_LAUNCH_CHECK();
}
void zero_f32(float* p, size_t n, cudaStream_t s) { GP_CUDA(cudaMemsetAsync(p, 0, n * sizeof(float), s)); }

void combine_fixed_point(const long long* const* acc, const float* scales, int ns, size_t n, double extra,
                         float* out, cudaStream_t s) {
  AccList a{};
  if (ns > 4) throw std::invalid_argument("at most 4 species");
  for (int i = 0; i < ns; ++i) {
    a.p[i] = acc[i];
    a.f[i] = double(scales[i]) * 0x1p-40 * extra;
  }
  launch_pdl(k_combine, dim3(grid1d(n)), dim3(256), 0, s, a, ns, n, out);
}

void combine_f64(const double* const* acc, int ns, size_t n, float* out, cudaStream_t s) {
  AccListD a{};
  if (ns > 4) throw std::invalid_argument("at most 4 species");
  for (int i = 0; i < ns; ++i) a.p[i] = acc[i];
  launch_pdl(k_combine_f64, dim3(grid1d(n)), dim3(256), 0, s, a, ns, n, out);
}

void fold_ghosts(float* rho, GridDims g, const int fbc[4], cudaStream_t s) {
  const int rows = g.ny + 1, cols = g.nx + 1;
  // exactly one x phase (0 or 2) and one y phase (1 or 3), in the reference's order
  if (fbc[0] != FBC_PERIODIC_C)
    launch_pdl(k_fold, dim3((rows + 127) / 128), dim3(128), 0, s, rho, g, fbc[0], fbc[1], fbc[2], fbc[3], 0);
  if (fbc[2] != FBC_PERIODIC_C)
    launch_pdl(k_fold, dim3((cols + 127) / 128), dim3(128), 0, s, rho, g, fbc[0], fbc[1], fbc[2], fbc[3], 1);
  if (fbc[0] == FBC_PERIODIC_C)
    launch_pdl(k_fold, dim3((rows + 127) / 128), dim3(128), 0, s, rho, g, fbc[0], fbc[1], fbc[2], fbc[3], 2);
  if (fbc[2] == FBC_PERIODIC_C)
    launch_pdl(k_fold, dim3((cols + 127) / 128), dim3(128), 0, s, rho, g, fbc[0], fbc[1], fbc[2], fbc[3], 3);
}

void build_rhs(const float* rho, GridDims g, PoissonLayout L, double* b, double* sums, cudaStream_t s) {
  const int n = (L.nkx + 1) * (L.nky + 1);
  GP_CUDA(cudaMemsetAsync(sums, 0, 2 * sizeof(double), s));
  launch_pdl(k_rhs, dim3(grid1d(n)), dim3(256), 0, s, rho, g, L, b, sums);
}

void vec_sums(const double* v, int n, double* sums, cudaStream_t s) {
  GP_CUDA(cudaMemsetAsync(sums, 0, 2 * sizeof(double), s));
  k_vec_sums<<<grid1d(n), 256, 0, s>>>(v, n, sums);
  GP_LAUNCH_CHECK();
}

void subtract_mean(double* v, int n, const double* sum, cudaStream_t s) {
  k_subtract_mean<<<grid1d(n), 256, 0, s>>>(v, n, sum);
  GP_LAUNCH_CHECK();
}

void phi_fill(const double* sol, GridDims g, PoissonLayout L, float dx, double cathode_pos, double* cathode_mean,
              double* phi, cudaStream_t s) {
  if (cathode_pos > 0.0) {
    const int col = int(cathode_pos / double(dx));
    if (col < 0 || col > L.nkx) throw std::invalid_argument("hollow-cathode position outside the solved grid");
    launch_pdl(k_cathode_mean, dim3(1), dim3(256), 0, s, sol, L, col, cathode_mean);
  }
  const size_t n = size_t(g.nx + 3) * (g.ny + 3);
  launch_pdl(k_phi_fill, dim3(grid1d(n)), dim3(256), 0, s, sol, g, L, dx, cathode_pos, cathode_mean, phi);
}

void gradient_energy(const double* phi, GridDims g, float dx, float dy, float* Ex, float* Ey, const float* jx,
                     const float* jy, double* sums, cudaStream_t s, float* Exp, float* Eyp) {
  const size_t n = size_t(g.nx + 2) * (g.ny + 1) + size_t(g.nx + 1) * (g.ny + 2);
  GP_CUDA(cudaMemsetAsync(sums, 0, 2 * sizeof(double), s));
  launch_pdl(k_gradient, dim3(grid1d(n)), dim3(256), 0, s, phi, g, dx, dy, Ex, Ey, jx, jy, sums, Exp, Eyp,
             field_pitch(g));
}

void probe(const double* phi, const float* Ex, const float* Ey, GridDims g, double* out3, cudaStream_t s) {
  launch_pdl(k_probe, dim3(1), dim3(1), 0, s, phi, Ex, Ey, g, out3);
}

}  // namespace kern
}  // namespace gample
