// multigrid.cu -- geometric multigrid Poisson solver (sm_100a).
#include "multigrid.hpp"
#include "pdl.cuh"

#include <algorithm>
#include <cfloat>
#include <mutex>
#include <cmath>
#include <stdexcept>

namespace gample {

namespace {

// Measured at 512^2 (solve ms per step): tiles of 32 x 16 points with 256
// threads 0.498, 32 x 8 with 512 threads 0.455 (16 x 16: 0.454, 64 x 8: 0.500,
// 32 x 8 with 1024 threads 0.472); the single-CTA kernel from 4096 points
// down 0.455, from 1024 points (63 x 64 in tiles) 0.438, from 256 points 0.596.
constexpr int kSmallPoints = 1024;       // levels at or below run in one CTA
constexpr int kMaxSmallLevels = 16;
constexpr int kDenseMax = 64;            // coarsest levels up to this size use a precomputed inverse
constexpr int TX = 32, TY = 8, HALO = 4;  // smoother tile and halo (4 half-sweeps)
constexpr int SW = TX + 2 * HALO, SH = TY + 2 * HALO;
constexpr int kSmoothThreads = 512;
constexpr int kSmallThreads = 1024;

// state words (FP64): see multigrid.hpp
enum {
  S_SUM = 0, S_SUM2, S_NORMB, S_REL, S_DONE, S_ITER, S_MEAN, S_REL0, S_ZQ, S_PQ, S_RP, S_PQOLD,
  S_ZAZ, S_RZ, S_RPO, S_PAZ, S_COUNT
};

// Partial sums of the flexible-CG passes: each block adds its sums into one
// of kSlots slots per quantity (block index mod kSlots), so at most
// 1/kSlots of the blocks queue on one address in the L2; the consumer sums
// the kSlots slots of a quantity with one warp.
constexpr int kSlots = 32;
enum { A_ZQ = 0, A_ZAZ, A_RZ, A_RPO, A_PAZ, A_SUM, A_SUM2, A_COUNT };

// Boundary treatment of a direction: Dirichlet (values outside are zero),
// periodic (wrap) or Neumann (mirror about the end node, i.e. the doubled
// off-diagonal of the Darwin operator, src/EMField.mm:527-560).
enum { BC_DIR = 0, BC_PER = 1, BC_NEU = 2 };

struct LevelDesc {
  int mx, my;
  int bx, by;
  float cx, cy, cd;
};

__host__ __device__ __forceinline__ bool wrap(int& i, int n, int b) {
  if (i >= 0 && i < n) return true;
  if (b == BC_DIR) return false;
  if (b == BC_PER) {
    i = ((i % n) + n) % n;
  } else {
    i = i < 0 ? -i : 2 * (n - 1) - i;
    if (i < 0 || i >= n) i = i < 0 ? 0 : n - 1;
  }
  return true;
}

// Weight of a node in the solvability condition of a singular level (the
// left null vector of the operator): 1/2 at each Neumann end, 1 elsewhere.
__host__ __device__ __forceinline__ float bc_weight(int i, int n, int b) {
  return (b == BC_NEU && (i == 0 || i == n - 1)) ? 0.5f : 1.0f;
}

__device__ __forceinline__ float ld(const float* u, const LevelDesc& d, int i, int j) {
  if (!wrap(i, d.mx, d.bx) || !wrap(j, d.my, d.by)) return 0.0f;
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

// Bilinear interpolation weights of fine index i from a coarse level
// (coarse I on fine 2I+1 for Dirichlet, 2I for periodic and Neumann).
__device__ __forceinline__ void interp1d(int i, int b, int mc, int& i0, float& w0, int& i1, float& w1) {
  if (b != BC_DIR) {
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

__device__ __forceinline__ float prolong_at(const float* uc, const LevelDesc& c, const LevelDesc& f, int i, int j) {
  int a0, a1, b0, b1;
  float wa0, wa1, wb0, wb1;
  interp1d(i, f.bx, c.mx, a0, wa0, a1, wa1);
  interp1d(j, f.by, c.my, b0, wb0, b1, wb1);
  return wb0 * (wa0 * uc[a0 + b0 * c.mx] + wa1 * uc[a1 + b0 * c.mx]) +
         wb1 * (wa0 * uc[a0 + b1 * c.mx] + wa1 * uc[a1 + b1 * c.mx]);
}

// Full-weighting restriction of the residual f - A u at coarse (I, J).
__device__ __forceinline__ float restrict_at(const float* u, const float* f, const LevelDesc& d, int I, int J) {
  const int fi = d.bx != BC_DIR ? 2 * I : 2 * I + 1;
  const int fj = d.by != BC_DIR ? 2 * J : 2 * J + 1;
  float s = 0.0f;
#pragma unroll
  for (int b = -1; b <= 1; ++b) {
    const float wb = b == 0 ? 0.5f : 0.25f;
#pragma unroll
    for (int a = -1; a <= 1; ++a) {
      const float wa = a == 0 ? 0.5f : 0.25f;
      int i = fi + a, j = fj + b;
      if (!wrap(i, d.mx, d.bx) || !wrap(j, d.my, d.by)) continue;
      const float au = d.cd * u[i + j * d.mx] + d.cx * (ld(u, d, i - 1, j) + ld(u, d, i + 1, j)) +
                       d.cy * (ld(u, d, i, j - 1) + ld(u, d, i, j + 1));
      s += wa * wb * (f[i + j * d.mx] - au);
    }
  }
  return s;
}

// ---------------------------------------------------------------- outer loop
// Start of a solve: the state words and the slots cleared (block 0), and,
// as AMGCL does for a zero right-hand side, x cleared (every block; the
// solve then returns at once).
__global__ void k_init(double* st, const double* sums_b, double* acc, double* x, int n) {
  grid_dependency_wait();
  grid_dependents_launch();
  const double nb = sqrt(sums_b[1] > 0 ? sums_b[1] : 0.0);
  const bool zero_rhs = nb < DBL_EPSILON;
  if (blockIdx.x == 0) {
    for (int i = threadIdx.x; i < A_COUNT * kSlots; i += blockDim.x) acc[i] = 0.0;
    if (threadIdx.x == 0) {
      for (int i = 0; i < S_COUNT; ++i) st[i] = 0.0;
      st[S_NORMB] = nb;
      if (zero_rhs) {
        st[S_DONE] = 2.0;
        st[S_REL] = nb;
      }
    }
  }
  if (zero_rhs)
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) x[k] = 0.0;
}

// (A v)_k in FP64 with the CSR row of src/EMField.mm:329-400 (diagonal,
// i-1, i+1, j-1, j+1); v(k) returns the vector's entry k.
template <class V>
__device__ __forceinline__ double apply_A(const kern::PoissonLayout& L, int k, int i, int j, int mx, V v) {
  const bool nx_ = L.fbc[0] == kern::FBC_NEUMANN_C, ny_ = L.fbc[2] == kern::FBC_NEUMANN_C;
  double ax = L.Cd * v(k);
  if (i > 0)
    ax += L.Cx * v(k - 1);
  else if (L.periodic_x)
    ax += L.Cx * v(k + L.nkx);
  else if (nx_ && L.nkx > 0)
    ax += L.Cx * v(k + 1);
  if (i < L.nkx)
    ax += L.Cx * v(k + 1);
  else if (L.periodic_x)
    ax += L.Cx * v(k - L.nkx);
  else if (nx_ && L.nkx > 0)
    ax += L.Cx * v(k - 1);
  if (j > 0)
    ax += L.Cy * v(k - mx);
  else if (L.periodic_y)
    ax += L.Cy * v(k + L.nky * mx);
  else if (ny_ && L.nky > 0)
    ax += L.Cy * v(k + mx);
  if (j < L.nky)
    ax += L.Cy * v(k + mx);
  else if (L.periodic_y)
    ax += L.Cy * v(k - L.nky * mx);
  else if (ny_ && L.nky > 0)
    ax += L.Cy * v(k - mx);
  return ax;
}

__device__ __forceinline__ double res_weight(const kern::PoissonLayout& L, int i, int j, int mx, int my) {
  const bool nx_ = L.fbc[0] == kern::FBC_NEUMANN_C, ny_ = L.fbc[2] == kern::FBC_NEUMANN_C;
  return double(bc_weight(i, mx, nx_ ? BC_NEU : BC_PER)) * bc_weight(j, my, ny_ ? BC_NEU : BC_PER);
}

// r = b - A x in FP64; stores r (r64, when given) and float(r) and
// accumulates sum w r, sum r^2; the last block to finish applies the
// stopping rule to the starting guess (AMGCL's ||r|| / ||b|| <= tol) and
// returns the counter to zero.
__global__ void k_residual64(const double* __restrict__ x, const double* __restrict__ b, kern::PoissonLayout L,
                             float* __restrict__ r32, double* __restrict__ r64, double* st, unsigned* ctr,
                             double tol, int maxiter, double wsum) {
  grid_dependency_wait();
  grid_dependents_launch();
  __shared__ double sh[32];
  __shared__ bool s_last;
  if (st[S_DONE] != 0.0) return;  // zero right-hand side: x was cleared
  const int mx = L.nkx + 1, my = L.nky + 1, n = mx * my;
  double s1 = 0.0, s2 = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int i = k % mx, j = k / mx;
    const bool nx_ = L.fbc[0] == kern::FBC_NEUMANN_C, ny_ = L.fbc[2] == kern::FBC_NEUMANN_C;
    const double ax = apply_A(L, k, i, j, mx, [&](int q) { return x[q]; });
    const double r = b[k] - ax;
    r32[k] = float(r);
    if (r64) r64[k] = r;
    const double w = double(bc_weight(i, mx, nx_ ? BC_NEU : BC_PER)) * bc_weight(j, my, ny_ ? BC_NEU : BC_PER);
    s1 += w * r;
    s2 += r * r;
  }
  s1 = block_sum(s1, sh);
  s2 = block_sum(s2, sh);
  if (threadIdx.x == 0) {
    atomicAdd(st + S_SUM, s1);
    atomicAdd(st + S_SUM2, s2);
    __threadfence();
    s_last = atomicAdd(ctr, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last && threadIdx.x == 0) {
    __threadfence();
    *ctr = 0u;
    const double sum = __ldcg(st + S_SUM), sum2 = __ldcg(st + S_SUM2);
    const double rel = sqrt(sum2 > 0 ? sum2 : 0.0) / st[S_NORMB];
    st[S_REL] = rel;
    st[S_REL0] = rel;
    if (!(rel > tol) || maxiter <= 0) {
      st[S_DONE] = 1.0;
    } else {
      st[S_ITER] = 1.0;
      st[S_MEAN] = sum / wsum;
    }
    st[S_SUM] = 0.0;
    st[S_SUM2] = 0.0;
  }
}

// Flexible conjugate gradients with the V-cycle as preconditioner (one
// retained direction, Notay's FCG(1)): z = M r, p = z + beta p_old with
// beta = -(z.q_old) / (p_old.q_old), q = A p, alpha = (r.p) / (p.q),
// x += alpha p, r -= alpha q. The orthogonalisation needs no symmetric or
// exact preconditioner, so the FP32 V-cycle serves as it is; the first
// iteration (S_ITER == 1) starts with p = z.
// Block sums of N values at once (one pair of barriers for all of them).
template <int N>
__device__ __forceinline__ void block_sums(double (&v)[N], double (*sh)[32]) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < N; ++a) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[a] += __shfl_xor_sync(0xffffffffu, v[a], o);
    if (lane == 0) sh[a][wid] = v[a];
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int a = 0; a < N; ++a) {
      double r = lane < int(blockDim.x >> 5) ? sh[a][lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
      v[a] = r;
    }
  }
  __syncthreads();
}

// The flexible-CG iteration in two passes. With q_old = A p_old,
//   p = z + beta p_old,  q = A p = A z + beta q_old,
//   p.q = z.Az + beta (z.q_old + p_old.Az) + beta^2 p_old.q_old,
//   r.p = r.z + beta r.p_old,
// so one pass over z, r, p_old, q_old gives every scalar (A z formed on the
// fly from z's neighbours; p_old.Az is kept apart from z.q_old because the
// operator is not symmetric with a Neumann direction), and a second pass
// updates p, q, x and r in place. Pass A: the dot products.
__global__ void k_fcg_dots(const float* __restrict__ z, const double* __restrict__ q_old,
                           const double* __restrict__ p_old, const double* __restrict__ r, kern::PoissonLayout L,
                           const double* st, double* acc) {
  grid_dependency_wait();
  grid_dependents_launch();
  __shared__ double sh[5][32];
  if (st[S_DONE] != 0.0) return;
  const bool first = st[S_ITER] == 1.0;  // p_old, q_old hold nothing of this solve yet
  const int mx = L.nkx + 1, my = L.nky + 1, n = mx * my;
  double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // z.q_old, z.Az, r.z, r.p_old, p_old.Az
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int i = k % mx, j = k / mx;
    const double zk = double(z[k]), rk = r[k];
    const double az = apply_A(L, k, i, j, mx, [&](int t) { return double(z[t]); });
    v[1] += zk * az;
    v[2] += rk * zk;
    if (!first) {
      const double po = p_old[k];
      v[0] += zk * q_old[k];
      v[3] += rk * po;
      v[4] += po * az;
    }
  }
  block_sums<5>(v, sh);
  if (threadIdx.x == 0) {
    const int slot = blockIdx.x % kSlots;
#pragma unroll
    for (int a = 0; a < 5; ++a) atomicAdd(acc + (A_ZQ + a) * kSlots + slot, v[a]);
  }
  (void)my;
}

// Sum of the kSlots slots of quantity a, by one full warp (every lane gets it).
__device__ __forceinline__ double slot_sum(const double* acc, int a) {
  double t = __ldcg(acc + a * kSlots + (threadIdx.x & 31));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  return t;
}

// The convergence test of one iteration (AMGCL's ||r|| / ||b|| <= tol or
// maxiter), run by one thread once every partial sum has arrived.
__device__ __forceinline__ void fcg_check(double* st, double pq, double tol, int maxiter, double wsum) {
  st[S_PQOLD] = pq;
  st[S_ZQ] = st[S_ZAZ] = st[S_RZ] = st[S_RPO] = st[S_PAZ] = 0.0;
  const double sum = __ldcg(st + S_SUM), sum2 = __ldcg(st + S_SUM2);
  const double rel = sqrt(sum2 > 0 ? sum2 : 0.0) / st[S_NORMB];
  st[S_REL] = rel;
  if (!(rel > tol) || st[S_ITER] >= double(maxiter)) {
    st[S_DONE] = 1.0;
  } else {
    st[S_ITER] += 1.0;
    st[S_MEAN] = sum / wsum;
  }
  st[S_SUM] = 0.0;
  st[S_SUM2] = 0.0;
}

// Pass B: p = z + beta p_old, q = A z + beta q_old (both in place), x +=
// alpha p, r -= alpha q with float(r) for the next V-cycle, kStepPoints
// points per thread. A thread loads its points' operands first, then the
// scalars from the slots of pass A (every block sums them in the same order,
// so all blocks use the same alpha and beta), so the two loads overlap. The
// last block to finish runs the convergence test, clears the slots for the
// next iteration and returns the counter to zero.
constexpr int kStepThreads = 256, kStepPoints = 2;
__global__ void __launch_bounds__(kStepThreads, 4) k_fcg_step(const float* __restrict__ z, double* __restrict__ p,
                                                           double* __restrict__ q, double* __restrict__ x,
                                                           double* __restrict__ r, float* __restrict__ r32,
                                                           kern::PoissonLayout L, double* st, double* acc,
                                                           unsigned* ctr, double tol, int maxiter, double wsum) {
  __shared__ double sh[2][32];
  __shared__ double s_sc[5];
  __shared__ bool s_last;
  grid_dependency_wait();
  grid_dependents_launch();
  // the stopping flag is tested after the operands and the slot sums are
  // loaded (uniform: every block sees the previous kernel's value)
  const bool done = st[S_DONE] != 0.0;
  const int mx = L.nkx + 1, my = L.nky + 1, n = mx * my;
  double az[kStepPoints], zk[kStepPoints], pk[kStepPoints], qk[kStepPoints], xk[kStepPoints], rk[kStepPoints];
#pragma unroll
  for (int t = 0; t < kStepPoints; ++t) {
    const int k = (blockIdx.x * kStepPoints + t) * kStepThreads + threadIdx.x;
    az[t] = zk[t] = pk[t] = qk[t] = xk[t] = rk[t] = 0.0;
    if (k < n) {
      az[t] = apply_A(L, k, k % mx, k / mx, mx, [&](int u) { return double(z[u]); });
      zk[t] = double(z[k]);
      pk[t] = p[k];
      qk[t] = q[k];
      xk[t] = x[k];
      rk[t] = r[k];
    }
  }
  if (threadIdx.x < 32) {
#pragma unroll
    for (int a = 0; a < 5; ++a) {
      const double t = slot_sum(acc, A_ZQ + a);
      if (threadIdx.x == 0) s_sc[a] = t;
    }
  }
  __syncthreads();
  if (done) return;
  const bool first = st[S_ITER] == 1.0;
  const double zq = s_sc[0], zaz = s_sc[1], rz = s_sc[2], rpo = s_sc[3], paz = s_sc[4];
  const double pq_old = st[S_PQOLD];
  const double beta = first ? 0.0 : -zq / pq_old;
  const double pq = zaz + (first ? 0.0 : beta * (zq + paz) + beta * beta * pq_old);
  const double rp = rz + (first ? 0.0 : beta * rpo);
  const double alpha = pq != 0.0 ? rp / pq : 0.0;
  double v[2] = {0.0, 0.0};  // sum w r, sum r^2
#pragma unroll
  for (int t = 0; t < kStepPoints; ++t) {
    const int k = (blockIdx.x * kStepPoints + t) * kStepThreads + threadIdx.x;
    if (k < n) {
      const double pn = first ? zk[t] : zk[t] + beta * pk[t];
      const double qn = first ? az[t] : az[t] + beta * qk[t];
      p[k] = pn;
      q[k] = qn;
      x[k] = xk[t] + alpha * pn;
      const double rn = rk[t] - alpha * qn;
      r[k] = rn;
      r32[k] = float(rn);
      v[0] += res_weight(L, k % mx, k / mx, mx, my) * rn;
      v[1] += rn * rn;
    }
  }
  block_sums<2>(v, sh);
  if (threadIdx.x == 0) {
    const int slot = blockIdx.x % kSlots;
    atomicAdd(acc + A_SUM * kSlots + slot, v[0]);
    atomicAdd(acc + A_SUM2 * kSlots + slot, v[1]);
    __threadfence();
    s_last = atomicAdd(ctr, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last && threadIdx.x < 32) {
    __threadfence();
    const double sum = slot_sum(acc, A_SUM), sum2 = slot_sum(acc, A_SUM2);
    __syncwarp();
#pragma unroll
    for (int a = 0; a < A_COUNT; ++a) acc[a * kSlots + threadIdx.x] = 0.0;
    if (threadIdx.x == 0) {
      *ctr = 0u;
      st[S_SUM] = sum;
      st[S_SUM2] = sum2;
      fcg_check(st, pq, tol, maxiter, wsum);
    }
  }
}

__global__ void k_sub_mean32(float* f, int n, const double* st) {
  grid_dependency_wait();
  grid_dependents_launch();
  if (st[S_DONE] != 0.0) return;
  const float m = float(st[S_MEAN]);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) f[k] -= m;
}

__global__ void k_sum64(const double* x, int n, double* out) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) s += x[k];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) atomicAdd(out, s);
}

__global__ void k_sub_mean64(double* x, int n, const double* sum) {
  const double m = sum[0] / double(n);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) x[k] -= m;
}

// ---------------------------------------------------------------- large levels
// Two red-black Gauss-Seidel iterations on a TX x TY tile, computed in shared
// memory with a 4-point halo (each half-sweep invalidates one ring), so the
// interior equals two global sweeps. PRE: starts from u = 0 (red, black, red,
// black). Otherwise adds the bilinear prolongation of the coarse correction
// first and sweeps black, red, black, red.
// The result goes to u_out: CTAs read their halos from u, so u itself must
// not change during the launch (u_out == u only when u is not read, PRE).
// Halo of the tile kernels: 4 points for the four half-sweeps; the
// pre-smoother keeps 2 more so that the residual on the tile's interior plus
// one ring (for the full-weighting restriction) is still exact.
// The finest level's post-smoother with DOTS also forms pass A of the
// flexible-CG iteration (z.q_old, z.Az, r.z, r.p_old, p_old.Az) on its tile:
// it keeps one more halo ring, so z is exact on the interior plus one ring
// and A z (FP64, the CSR coefficients of the fine system) is formed in
// shared memory.
template <bool PRE, bool DOTS = false>
constexpr int tile_halo() {
  return PRE ? HALO + 2 : DOTS ? HALO + 1 : HALO;
}

// Operands of pass A for the fused post-smoother of the finest level.
struct FcgDotsIn {
  const double* r;
  const double* p_old;
  const double* q_old;
  double* acc;
  double cx, cy, cd;
};

template <bool PRE, bool DOTS = false>
__global__ void __launch_bounds__(kSmoothThreads, 4) k_smooth_tile(const float* u, float* u_out,
                                                                const float* __restrict__ f, LevelDesc d,
                                                                const float* __restrict__ uc, LevelDesc c,
                                                                const double* st, float* __restrict__ fc_out,
                                                                FcgDotsIn fd = FcgDotsIn{}) {
  grid_dependency_wait();
  grid_dependents_launch();
  static_assert(!(PRE && DOTS), "pass A belongs to the post-smoother");
  constexpr int HL = tile_halo<PRE, DOTS>(), W = TX + 2 * HL, H = TY + 2 * HL;
  __shared__ float su[H][W + 1];
  __shared__ float sf[H][W + 1];
  __shared__ unsigned char s_in[H][W];
  // the stopping flag and the tile are loaded together; the (uniform) test
  // comes after the tile's loads are issued
  const bool done = st[S_DONE] != 0.0;
  const int x0 = blockIdx.x * TX - HL, y0 = blockIdx.y * TY - HL;
  // pass A operands of this thread's interior point, loaded before the sweeps
  static_assert(TX * TY <= kSmoothThreads, "one interior point per thread");
  double d_r = 0.0, d_p = 0.0, d_q = 0.0;
  bool d_first = false;
  if constexpr (DOTS) {
    d_first = st[S_ITER] == 1.0;  // p_old, q_old hold nothing of this solve yet
    const int gi = x0 + HL + int(threadIdx.x) % TX, gj = y0 + HL + int(threadIdx.x) / TX;
    if (threadIdx.x < TX * TY && gi < d.mx && gj < d.my) {
      const int k = gi + gj * d.mx;
      d_r = fd.r[k];
      if (!d_first) {
        d_p = fd.p_old[k];
        d_q = fd.q_old[k];
      }
    }
  }
  for (int e = threadIdx.x; e < W * H; e += kSmoothThreads) {
    const int li = e % W, lj = e / W;
    int gi = x0 + li, gj = y0 + lj;
    const bool inside = wrap(gi, d.mx, d.bx) && wrap(gj, d.my, d.by);
    float uv = 0.0f, fv = 0.0f;
    if (inside) {
      fv = f[gi + gj * d.mx];
      if (!PRE) uv = u[gi + gj * d.mx] + prolong_at(uc, c, d, gi, gj);
    }
    su[lj][li] = uv;
    sf[lj][li] = fv;
    s_in[lj][li] = inside ? 1 : 0;
  }
  if (done) return;
  __syncthreads();
  const float inv = 1.0f / d.cd;
#pragma unroll
  for (int hs = 0; hs < 4; ++hs) {
    const int color = PRE ? (hs & 1) : 1 - (hs & 1);
    // points of this color in [1, W-2] x [1, H-2]
    for (int e = threadIdx.x; e < (W - 2) * (H - 2) / 2 + H; e += kSmoothThreads) {
      const int lj = 1 + e / ((W - 2) / 2);
      if (lj > H - 2) break;
      const int k = e % ((W - 2) / 2);
      // global parity (x0 + li + y0 + lj) & 1 == color
      const int par = (x0 + y0 + lj + 1) & 1;  // parity of li = 1
      const int li = 1 + 2 * k + ((par ^ color) & 1);
      if (li > W - 2 || !s_in[lj][li]) continue;
      const float s = d.cx * (su[lj][li - 1] + su[lj][li + 1]) + d.cy * (su[lj - 1][li] + su[lj + 1][li]);
      su[lj][li] = (sf[lj][li] - s) * inv;
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < TX * TY; e += kSmoothThreads) {
    const int li = HL + e % TX, lj = HL + e / TX;
    const int gi = x0 + li, gj = y0 + lj;
    if (gi < d.mx && gj < d.my) u_out[gi + gj * d.mx] = su[lj][li];
  }
  if constexpr (DOTS) {
    // Outside a Dirichlet wall su is 0 (the CSR row has no entry there);
    // periodic and mirrored neighbours were loaded as such.
    __shared__ double sh[5][32];
    double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // z.q_old, z.Az, r.z, r.p_old, p_old.Az
    const int li = HL + int(threadIdx.x) % TX, lj = HL + int(threadIdx.x) / TX;
    if (threadIdx.x < TX * TY && x0 + li < d.mx && y0 + lj < d.my) {
      const double zk = double(su[lj][li]);
      const double az = fd.cd * zk + fd.cx * double(su[lj][li - 1]) + fd.cx * double(su[lj][li + 1]) +
                        fd.cy * double(su[lj - 1][li]) + fd.cy * double(su[lj + 1][li]);
      v[1] = zk * az;
      v[2] = d_r * zk;
      if (!d_first) {
        v[0] = zk * d_q;
        v[3] = d_r * d_p;
        v[4] = d_p * az;
      }
    }
    block_sums<5>(v, sh);
    if (threadIdx.x == 0) {
      const int slot = (blockIdx.x + blockIdx.y * gridDim.x) % kSlots;
#pragma unroll
      for (int a = 0; a < 5; ++a) atomicAdd(fd.acc + (A_ZQ + a) * kSlots + slot, v[a]);
    }
  }
  if constexpr (PRE) {
    if (!fc_out) return;
    // residual r = f - A u on the interior plus one ring (into sr), then the
    // full-weighting restriction of the coarse points whose centre this tile owns
    __shared__ float sr[TY + 2][TX + 2];
    for (int e = threadIdx.x; e < (TX + 2) * (TY + 2); e += kSmoothThreads) {
      const int li = HL - 1 + e % (TX + 2), lj = HL - 1 + e / (TX + 2);
      float r = 0.0f;
      if (s_in[lj][li])
        r = sf[lj][li] - (d.cd * su[lj][li] + d.cx * (su[lj][li - 1] + su[lj][li + 1]) +
                          d.cy * (su[lj - 1][li] + su[lj + 1][li]));
      sr[lj - (HL - 1)][li - (HL - 1)] = r;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < (TX / 2) * (TY / 2); e += kSmoothThreads) {
      const int I = blockIdx.x * (TX / 2) + e % (TX / 2), J = blockIdx.y * (TY / 2) + e / (TX / 2);
      if (I >= c.mx || J >= c.my) continue;
      const int fi = d.bx != BC_DIR ? 2 * I : 2 * I + 1, fj = d.by != BC_DIR ? 2 * J : 2 * J + 1;
      const int li = fi - x0 - (HL - 1), lj = fj - y0 - (HL - 1);  // in sr
      float v = 0.0f;
#pragma unroll
      for (int b = -1; b <= 1; ++b) {
        const float wb = b == 0 ? 0.5f : 0.25f;
#pragma unroll
        for (int a = -1; a <= 1; ++a) v += (a == 0 ? 0.5f : 0.25f) * wb * sr[lj + b][li + a];
      }
      fc_out[I + J * c.mx] = v;
    }
  }
}

__global__ void k_restrict(const float* __restrict__ u, const float* __restrict__ f, LevelDesc d, float* __restrict__ fc,
                           LevelDesc c, const double* st) {
  grid_dependency_wait();
  grid_dependents_launch();
  if (st[S_DONE] != 0.0) return;
  const int n = c.mx * c.my;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    fc[k] = restrict_at(u, f, d, k % c.mx, k / c.mx);
}

// Generic (untiled) red-black half sweep, used for large levels whose shape
// does not fit the tile kernel.
__global__ void k_smooth_generic(float* __restrict__ u, const float* __restrict__ f, LevelDesc d, int color,
                                 const double* st) {
  grid_dependency_wait();
  grid_dependents_launch();
  if (st[S_DONE] != 0.0) return;
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

__global__ void k_prolong_generic(const float* __restrict__ uc, LevelDesc c, float* __restrict__ uf, LevelDesc d,
                                  const double* st) {
  grid_dependency_wait();
  grid_dependents_launch();
  if (st[S_DONE] != 0.0) return;
  const int n = d.mx * d.my;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    uf[k] += prolong_at(uc, c, d, k % d.mx, k / d.mx);
}

__global__ void k_zero32(float* u, int n, const double* st) {
  grid_dependency_wait();
  grid_dependents_launch();
  if (st[S_DONE] != 0.0) return;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) u[k] = 0.0f;
}


// ---------------------------------------------------------------- small levels
struct SmallLevels {
  int count;  // levels ls .. ls+count-1
  LevelDesc d[kMaxSmallLevels];
  int off[kMaxSmallLevels];  // float offset of u; f at +n, r at +2n
  int cg_off;                // 3 CG vectors of the coarsest level
  const float* cinv;         // dense inverse of the coarsest operator (nullptr: CG), staged at cg_off
};

// Small-level helpers for the single CTA of kSmallThreads = 32 x kRows
// threads: thread (tx, ty) takes columns tx, tx + 32, ... of rows ty, ty + kRows,
// ... (no integer division), and neighbours are read with explicit wraps.
constexpr int kRows = kSmallThreads / 32;

__device__ __forceinline__ float nb_sum(const float* u, const LevelDesc& d, int i, int j) {
  const int k = i + j * d.mx;
  const int ox = d.mx > 1 ? 1 : 0, oy = d.my > 1 ? d.mx : 0;  // Neumann mirror neighbours
  const float l = i > 0 ? u[k - 1] : (d.bx == BC_PER ? u[k + d.mx - 1] : d.bx == BC_NEU ? u[k + ox] : 0.0f);
  const float r = i < d.mx - 1 ? u[k + 1] : (d.bx == BC_PER ? u[k - d.mx + 1] : d.bx == BC_NEU ? u[k - ox] : 0.0f);
  const float b = j > 0 ? u[k - d.mx] : (d.by == BC_PER ? u[k + (d.my - 1) * d.mx] : d.by == BC_NEU ? u[k + oy] : 0.0f);
  const float t = j < d.my - 1 ? u[k + d.mx]
                               : (d.by == BC_PER ? u[k - (d.my - 1) * d.mx] : d.by == BC_NEU ? u[k - oy] : 0.0f);
  return d.cx * (l + r) + d.cy * (b + t);
}

__device__ __forceinline__ void sb_smooth(float* u, const float* f, const LevelDesc& d, int color) {
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int hx = (d.mx + 1) >> 1;
  const float inv = 1.0f / d.cd;
  for (int j = ty; j < d.my; j += kRows) {
    const int par = (j + color) & 1;
    for (int h = tx; h < hx; h += 32) {
      const int i = 2 * h + par;
      if (i < d.mx) u[i + j * d.mx] = (f[i + j * d.mx] - nb_sum(u, d, i, j)) * inv;
    }
  }
  __syncthreads();
}

// The first red half-sweep from u = 0: every neighbour is zero, so the red
// points become f / cd and the black ones stay zero (the same values as
// zeroing u and sweeping, in one pass).
__device__ __forceinline__ void sb_first_red(float* u, const float* f, const LevelDesc& d) {
  const float inv = 1.0f / d.cd;
  for (int k = threadIdx.x; k < d.mx * d.my; k += kSmallThreads) {
    const int i = k % d.mx, j = k / d.mx;
    u[k] = ((i + j) & 1) == 0 ? (f[k] - 0.0f) * inv : 0.0f;
  }
  __syncthreads();
}

// r = f - A u, then full weighting of r onto the coarse right-hand side.
__device__ __forceinline__ void sb_restrict(const float* u, const float* f, float* r, const LevelDesc& d, float* fc,
                            const LevelDesc& c) {
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int j = ty; j < d.my; j += kRows)
    for (int i = tx; i < d.mx; i += 32) {
      const int k = i + j * d.mx;
      r[k] = f[k] - (d.cd * u[k] + nb_sum(u, d, i, j));
    }
  __syncthreads();
  for (int J = ty; J < c.my; J += kRows)
    for (int I = tx; I < c.mx; I += 32) {
      const int fi = d.bx != BC_DIR ? 2 * I : 2 * I + 1;
      const int fj = d.by != BC_DIR ? 2 * J : 2 * J + 1;
      float s = 0.0f;
#pragma unroll
      for (int b = -1; b <= 1; ++b) {
        int j = fj + b;
        if (!wrap(j, d.my, d.by)) continue;
        const float wb = b == 0 ? 0.5f : 0.25f;
#pragma unroll
        for (int a = -1; a <= 1; ++a) {
          int i = fi + a;
          if (!wrap(i, d.mx, d.bx)) continue;
          s += (a == 0 ? 0.5f : 0.25f) * wb * r[i + j * d.mx];
        }
      }
      fc[I + J * c.mx] = s;
    }
  __syncthreads();
}

__device__ __forceinline__ void sb_prolong_add(float* u, const LevelDesc& d, const float* uc, const LevelDesc& c) {
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int j = ty; j < d.my; j += kRows)
    for (int i = tx; i < d.mx; i += 32) u[i + j * d.mx] += prolong_at(uc, c, d, i, j);
  __syncthreads();
}

// u = M (f - mean f) with M (in shared memory) the inverse of the coarsest
// operator (of A + a 11^T for the doubly periodic one, whose zero-mean
// solutions it returns).
__device__ __forceinline__ void sm_dense_solve(float* u, const float* f, const LevelDesc& d, const float* M, double* sh,
                               double* sval) {
  const int n = d.mx * d.my;
  const bool singular = d.bx != BC_DIR && d.by != BC_DIR;
  float mean = 0.0f;
  if (singular) {  // project f onto the range: subtract its weighted mean
    double s = 0.0, w = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      const double wk = double(bc_weight(k % d.mx, d.mx, d.bx)) * bc_weight(k / d.mx, d.my, d.by);
      s += wk * f[k];
      w += wk;
    }
    s = block_sum(s, sh);
    w = block_sum(w, sh);
    if (threadIdx.x == 0) *sval = s / w;
    __syncthreads();
    mean = float(*sval);
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    float acc = 0.0f;
    for (int j = 0; j < n; ++j) acc = fmaf(M[i * n + j], f[j] - mean, acc);
    u[i] = acc;
  }
  __syncthreads();
  if (singular) {
    double s = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) s += u[k];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) *sval = s / n;
    __syncthreads();
    const float m = float(*sval);
    for (int k = threadIdx.x; k < n; k += blockDim.x) u[k] -= m;
    __syncthreads();
  }
}

// CG on (-W A) u = -W f (shared memory), W = the solvability weights (1/2 at
// Neumann ends, making the operator symmetric; 1 otherwise). A singular
// level (no Dirichlet direction) is solved in its range: f is projected with
// the weights and u returned with zero mean.
__device__ __forceinline__ void sm_coarse_cg(float* u, const float* f, const LevelDesc& d, float* work, double* sh, double* sval) {
  const int n = d.mx * d.my;
  float* r = work;
  float* p = work + n;
  float* q = work + 2 * n;
  const bool singular = d.bx != BC_DIR && d.by != BC_DIR;
  auto wt = [&](int k) { return bc_weight(k % d.mx, d.mx, d.bx) * bc_weight(k / d.mx, d.my, d.by); };
  double mean = 0.0;
  if (singular) {
    double s = 0.0, w = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      s += double(wt(k)) * f[k];
      w += wt(k);
    }
    s = block_sum(s, sh);
    w = block_sum(w, sh);
    if (threadIdx.x == 0) *sval = s / w;
    __syncthreads();
    mean = *sval;
  }
  double rr = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const float v = -wt(k) * (f[k] - float(mean));
    u[k] = 0.0f;
    r[k] = v;
    p[k] = v;
    rr += double(v) * v;
  }
  rr = block_sum(rr, sh);
  if (threadIdx.x == 0) *sval = rr;
  __syncthreads();
  rr = *sval;
  const double stop = 1e-10 * rr;
  const int maxit = 2 * n + 10 < 2000 ? 2 * n + 10 : 2000;
  for (int it = 0; it < maxit && rr > stop && rr > 0.0; ++it) {
    double pq = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      const int i = k % d.mx, j = k / d.mx;
      const float ap = d.cd * p[k] + d.cx * (ld(p, d, i - 1, j) + ld(p, d, i + 1, j)) +
                       d.cy * (ld(p, d, i, j - 1) + ld(p, d, i, j + 1));
      q[k] = -wt(k) * ap;
      pq += double(p[k]) * double(q[k]);
    }
    pq = block_sum(pq, sh);
    if (threadIdx.x == 0) *sval = pq;
    __syncthreads();
    pq = *sval;
    if (!(pq > 0.0)) break;
    const float alpha = float(rr / pq);
    double rn = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      u[k] += alpha * p[k];
      r[k] -= alpha * q[k];
      rn += double(r[k]) * r[k];
    }
    rn = block_sum(rn, sh);
    if (threadIdx.x == 0) *sval = rn;
    __syncthreads();
    rn = *sval;
    const float beta = float(rn / rr);
    rr = rn;
    for (int k = threadIdx.x; k < n; k += blockDim.x) p[k] = r[k] + beta * p[k];
    __syncthreads();
  }
  if (singular) {
    double s = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) s += u[k];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) *sval = s / n;
    __syncthreads();
    const float m = float(*sval);
    for (int k = threadIdx.x; k < n; k += blockDim.x) u[k] -= m;
    __syncthreads();
  }
}

// The V-cycle of every small level in one CTA: f of the first small level is
// read from global memory, its correction u written back (and added to the
// FP64 solution when it is the finest level).
// BX, BY: the boundary type of each direction (the same on every level), a
// compile-time constant in the stencil code.
template <int BX, int BY>
__global__ void __launch_bounds__(kSmallThreads) k_small_vcycle(SmallLevels S, const float* __restrict__ f_in,
                                                                float* __restrict__ u_out, double* x, int nu_pre,
                                                                int nu_post, const double* st) {
  grid_dependency_wait();
  grid_dependents_launch();
  extern __shared__ float sm[];
  __shared__ double sh[32];
  __shared__ double sval;
  const bool done = st[S_DONE] != 0.0;  // tested once the level data's loads are issued
  auto level = [&](int l) {
    LevelDesc d = S.d[l];
    d.bx = BX;
    d.by = BY;
    return d;
  };
  const LevelDesc d0 = level(0);
  const int n0 = d0.mx * d0.my;
  for (int k = threadIdx.x; k < n0; k += blockDim.x) sm[S.off[0] + n0 + k] = f_in[k];
  if (S.cinv) {
    const LevelDesc& c = S.d[S.count - 1];
    const int nn = c.mx * c.my * c.mx * c.my;
    for (int k = threadIdx.x; k < nn; k += blockDim.x) sm[S.cg_off + k] = __ldg(S.cinv + k);
  }
  if (done) return;
  __syncthreads();
  const int last = S.count - 1;
  for (int l = 0; l < last; ++l) {
    const LevelDesc d = level(l);
    const LevelDesc c = level(l + 1);
    const int n = d.mx * d.my;
    float* u = sm + S.off[l];
    for (int it = 0; it < nu_pre; ++it) {
      if (it == 0)
        sb_first_red(u, u + n, d);
      else
        sb_smooth(u, u + n, d, 0);
      sb_smooth(u, u + n, d, 1);
    }
    if (nu_pre == 0) {
      for (int k = threadIdx.x; k < n; k += kSmallThreads) u[k] = 0.0f;
      __syncthreads();
    }
    sb_restrict(u, u + n, u + 2 * n, d, sm + S.off[l + 1] + c.mx * c.my, c);
  }
  {
    const LevelDesc d = level(last);
    float* u = sm + S.off[last];
    if (S.cinv) {
      sm_dense_solve(u, u + d.mx * d.my, d, sm + S.cg_off, sh, &sval);
    } else {
      sm_coarse_cg(u, u + d.mx * d.my, d, sm + S.cg_off, sh, &sval);
      __syncthreads();
    }
  }
  for (int l = last - 1; l >= 0; --l) {
    const LevelDesc d = level(l);
    const LevelDesc c = level(l + 1);
    const int n = d.mx * d.my;
    float* u = sm + S.off[l];
    sb_prolong_add(u, d, sm + S.off[l + 1], c);
    for (int it = 0; it < nu_post; ++it) {
      sb_smooth(u, u + n, d, 1);
      sb_smooth(u, u + n, d, 0);
    }
  }
  for (int k = threadIdx.x; k < n0; k += blockDim.x) {
    const float v = sm[S.off[0] + k];
    u_out[k] = v;
    if (x) x[k] += double(v);
  }
}

using SmallKernel = void (*)(SmallLevels, const float*, float*, double*, int, int, const double*);
SmallKernel small_kernel(int bx, int by) {
  static const SmallKernel table[9] = {
      k_small_vcycle<BC_DIR, BC_DIR>, k_small_vcycle<BC_DIR, BC_PER>, k_small_vcycle<BC_DIR, BC_NEU>,
      k_small_vcycle<BC_PER, BC_DIR>, k_small_vcycle<BC_PER, BC_PER>, k_small_vcycle<BC_PER, BC_NEU>,
      k_small_vcycle<BC_NEU, BC_DIR>, k_small_vcycle<BC_NEU, BC_PER>, k_small_vcycle<BC_NEU, BC_NEU>};
  return table[bx * 3 + by];
}

int blocks_for(int n) {
  long long b = ((long long)n + 255) / 256;
  if (b < 1) b = 1;
  return int(b < 2368 ? b : 2368);
}

// Grid of the kernels that end in a global FP64 reduction: four CTAs per SM,
// so that each adds its partial sums once (the adds to one address are
// serialised in the L2) and each thread covers a few points (measured at
// 512^2: 2, 4, 6, 8 CTAs per SM give 0.498, 0.487, 0.499, 0.531 ms of solve
// per step).
int reduce_blocks(int n) {
  static int cap = 0;
  if (!cap) {
    int dev = 0, sms = 0;
    GP_CUDA(cudaGetDevice(&dev));
    GP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    cap = 4 * sms;
  }
  const int b = blocks_for(n);
  return b < cap ? b : cap;
}

LevelDesc desc(const PoissonMG::Level& l) { return LevelDesc{l.mx, l.my, l.bx, l.by, l.cx, l.cy, l.cd}; }

bool can_coarsen(int n, int b) { return b == BC_PER ? (n >= 4 && n % 2 == 0) : (n >= 3 && n % 2 == 1); }
int coarser(int n, int b) { return b == BC_PER ? n / 2 : b == BC_NEU ? (n + 1) / 2 : (n - 1) / 2; }
bool tiled(const PoissonMG::Level& l) {
  return l.mx >= SW && l.my >= SH && (l.bx != BC_PER || l.mx % 2 == 0) && (l.by != BC_PER || l.my % 2 == 0);
}
// the pre-smoother with the fused residual + restriction (wider halo)
bool tiled_pre(const PoissonMG::Level& l) {
  return tiled(l) && l.mx >= SW + 4 && l.my >= SH + 4;
}
// the finest post-smoother with the fused pass A of the flexible CG (one more ring)
bool tiled_dots(const PoissonMG::Level& l) {
  return tiled(l) && l.mx >= SW + 2 && l.my >= SH + 2;
}
int bc_code(const kern::PoissonLayout& L, bool x) {
  if (x ? L.periodic_x : L.periodic_y) return BC_PER;
  return L.fbc[x ? 0 : 2] == kern::FBC_NEUMANN_C ? BC_NEU : BC_DIR;
}

}  // namespace

PoissonMG::PoissonMG(const kern::PoissonLayout& L, int nu_pre, int nu_post)
    : L_(L), nu_pre_(nu_pre), nu_post_(nu_post), state_(S_COUNT, true), host_(S_COUNT) {
  if (!((L.fbc[0] == kern::FBC_PERIODIC_C) == (L.fbc[1] == kern::FBC_PERIODIC_C)) ||
      !((L.fbc[2] == kern::FBC_PERIODIC_C) == (L.fbc[3] == kern::FBC_PERIODIC_C)))
    throw std::invalid_argument("periodic field boundaries must be set on both walls of a direction");
  if (L.fbc[0] != L.fbc[1] || L.fbc[2] != L.fbc[3])
    throw std::invalid_argument("both walls of a direction must have the same boundary type");
  const int bx = bc_code(L, true), by = bc_code(L, false);
  bx_ = bx;
  by_ = by;
  int mx = L.nkx + 1, my = L.nky + 1;
  if (mx < 1 || my < 1) throw std::invalid_argument("empty Poisson system");
  n_ = mx * my;
  float cx = float(L.Cx), cy = float(L.Cy);
  for (;;) {
    Level lv;
    lv.mx = mx;
    lv.my = my;
    lv.bx = bx;
    lv.by = by;
    lv.cx = cx;
    lv.cy = cy;
    lv.cd = -2.0f * (cx + cy);
    lv.u.resize(size_t(mx) * my, true);
    lv.u2.resize(size_t(mx) * my, true);
    lv.f.resize(size_t(mx) * my, true);
    lv_.push_back(std::move(lv));
    if (!(can_coarsen(mx, bx) && can_coarsen(my, by))) break;
    if (size_t(mx) * my <= size_t(kDenseMax)) break;  // solved by its dense inverse
    mx = coarser(mx, bx);
    my = coarser(my, by);
    cx *= 0.25f;
    cy *= 0.25f;
  }
  // first level small enough for the single-CTA kernel (all levels below it too)
  ls_ = int(lv_.size());
  for (int l = 0; l < int(lv_.size()); ++l)
    if (size_t(lv_[l].mx) * lv_[l].my <= size_t(kSmallPoints) && int(lv_.size()) - l <= kMaxSmallLevels) {
      ls_ = l;
      break;
    }
  if (ls_ == int(lv_.size())) ls_ = int(lv_.size()) - 1;  // coarsest larger than kSmallPoints: one-level CG kernel
  size_t floats = 0;
  for (int l = ls_; l < int(lv_.size()); ++l) floats += 3 * size_t(lv_[l].mx) * lv_[l].my;
  const Level& c = lv_.back();
  const size_t ncoarse = size_t(c.mx) * c.my;
  floats += ncoarse <= size_t(kDenseMax) ? std::max(3 * ncoarse, ncoarse * ncoarse) : 3 * ncoarse;  // inverse or CG
  small_smem_ = floats * sizeof(float);
  int dev = 0, maxsm = 0;
  GP_CUDA(cudaGetDevice(&dev));
  GP_CUDA(cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (small_smem_ + 2048 > size_t(maxsm))
    throw std::invalid_argument("coarsest multigrid level too large (grid dimensions do not coarsen)");
  // The attribute is per function and shared by every solver in the process
  // (ensemble members run concurrently): allow the device's maximum once.
  static std::once_flag once;
  std::call_once(once, [maxsm] {
    for (int b = 0; b < 9; ++b) {
      const SmallKernel k = small_kernel(b / 3, b % 3);
      cudaFuncAttributes fa{};
      GP_CUDA(cudaFuncGetAttributes(&fa, k));
      GP_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm - int(fa.sharedSizeBytes)));
    }
  });
  r64_.resize(size_t(n_), true);
  q_.resize(size_t(n_), true);
  ctr_.resize(1, true);
  acc_.resize(size_t(A_COUNT) * kSlots, true);
  p_[0].resize(size_t(n_), true);
  // Dense inverse of the coarsest operator (FP64 Gauss-Jordan, stored FP32);
  // a singular one (no Dirichlet direction) is regularised as A + a 1 w^T
  // with w its left null vector and a = |cd| / n, whose inverse returns the
  // w-orthogonal solution for a right-hand side with w^T f = 0.
  const int nc = c.mx * c.my;
  singular_ = bx != BC_DIR && by != BC_DIR;
  wsum_ = 0.0;
  for (int j = 0; j < my_top(); ++j)
    for (int i = 0; i < mx_top(); ++i) wsum_ += double(bc_weight(i, mx_top(), bx)) * bc_weight(j, my_top(), by);
  if (nc <= kDenseMax) {
    std::vector<double> A(size_t(nc) * nc, 0.0), I(size_t(nc) * nc, 0.0);
    for (int j = 0; j < c.my; ++j)
      for (int i = 0; i < c.mx; ++i) {
        const int k = i + j * c.mx;
        A[size_t(k) * nc + k] += c.cd;
        const int di[4] = {-1, 1, 0, 0}, dj[4] = {0, 0, -1, 1};
        for (int q = 0; q < 4; ++q) {
          int ii = i + di[q], jj = j + dj[q];
          if (!wrap(ii, c.mx, c.bx) || !wrap(jj, c.my, c.by)) continue;
          A[size_t(k) * nc + ii + jj * c.mx] += q < 2 ? c.cx : c.cy;
        }
      }
    if (singular_)
      for (int r = 0; r < nc; ++r)
        for (int q = 0; q < nc; ++q)
          A[size_t(r) * nc + q] +=
              std::fabs(double(c.cd)) / nc * bc_weight(q % c.mx, c.mx, c.bx) * bc_weight(q / c.mx, c.my, c.by);
    for (int k = 0; k < nc; ++k) I[size_t(k) * nc + k] = 1.0;
    for (int col = 0; col < nc; ++col) {
      int piv = col;
      for (int r = col + 1; r < nc; ++r)
        if (std::fabs(A[size_t(r) * nc + col]) > std::fabs(A[size_t(piv) * nc + col])) piv = r;
      if (std::fabs(A[size_t(piv) * nc + col]) < 1e-300) throw std::runtime_error("singular coarsest multigrid level");
      for (int q = 0; q < nc; ++q) {
        std::swap(A[size_t(col) * nc + q], A[size_t(piv) * nc + q]);
        std::swap(I[size_t(col) * nc + q], I[size_t(piv) * nc + q]);
      }
      const double inv = 1.0 / A[size_t(col) * nc + col];
      for (int q = 0; q < nc; ++q) {
        A[size_t(col) * nc + q] *= inv;
        I[size_t(col) * nc + q] *= inv;
      }
      for (int r = 0; r < nc; ++r) {
        if (r == col) continue;
        const double fct = A[size_t(r) * nc + col];
        if (fct == 0.0) continue;
        for (int q = 0; q < nc; ++q) {
          A[size_t(r) * nc + q] -= fct * A[size_t(col) * nc + q];
          I[size_t(r) * nc + q] -= fct * I[size_t(col) * nc + q];
        }
      }
    }
    std::vector<float> M(I.begin(), I.end());
    coarse_inv_.resize(M.size());
    GP_CUDA(cudaMemcpy(coarse_inv_.get(), M.data(), M.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
}

bool PoissonMG::vcycle(cudaStream_t s, bool with_dots) {
  double* st = state_.get();
  bool fused_dots = false;
  const int nl = int(lv_.size());
  // descent over the large levels
  for (int l = 0; l < ls_; ++l) {
    Level& a = lv_[l];
    Level& b = lv_[l + 1];
    const LevelDesc d = desc(a);
    if (tiled_pre(a) && nu_pre_ == 2) {  // smoothing, residual and restriction in one launch
      dim3 grid((a.mx + TX - 1) / TX, (a.my + TY - 1) / TY);
      launch_pdl(k_smooth_tile<true>, grid, dim3(kSmoothThreads), 0, s, a.u.get(), a.u.get(), a.f.get(), d, nullptr, desc(b), st, b.f.get(), FcgDotsIn{});
      continue;
    } else if (tiled(a) && nu_pre_ == 2) {
      dim3 grid((a.mx + TX - 1) / TX, (a.my + TY - 1) / TY);
      launch_pdl(k_smooth_tile<true>, grid, dim3(kSmoothThreads), 0, s, a.u.get(), a.u.get(), a.f.get(), d, nullptr, d, st, nullptr, FcgDotsIn{});
    } else {
      launch_pdl(k_zero32, dim3(blocks_for(a.mx * a.my)), dim3(256), 0, s, a.u.get(), a.mx * a.my, st);
      for (int it = 0; it < nu_pre_; ++it) {
        launch_pdl(k_smooth_generic, dim3(blocks_for((a.mx + 1) / 2 * a.my)), dim3(256), 0, s, a.u.get(), a.f.get(), d, 0, st);
        launch_pdl(k_smooth_generic, dim3(blocks_for((a.mx + 1) / 2 * a.my)), dim3(256), 0, s, a.u.get(), a.f.get(), d, 1, st);
      }
    }
    launch_pdl(k_restrict, dim3(blocks_for(b.mx * b.my)), dim3(256), 0, s, a.u.get(), a.f.get(), d, b.f.get(), desc(b), st);
  }
  // all small levels in one CTA
  {
    SmallLevels S{};
    S.count = nl - ls_;
    size_t off = 0;
    for (int l = ls_; l < nl; ++l) {
      S.d[l - ls_] = desc(lv_[l]);
      S.off[l - ls_] = int(off);
      off += 3 * size_t(lv_[l].mx) * lv_[l].my;
    }
    S.cg_off = int(off);
    S.cinv = coarse_inv_.size() ? coarse_inv_.get() : nullptr;
    launch_pdl(small_kernel(bx_, by_), dim3(1), dim3(kSmallThreads), small_smem_, s, S, lv_[ls_].f.get(), lv_[ls_].u.get(), nullptr, nu_pre_, nu_post_, st);
    lv_[ls_].result_in_u2 = false;
  }
  // ascent
  for (int l = ls_ - 1; l >= 0; --l) {
    Level& a = lv_[l];
    Level& b = lv_[l + 1];
    const LevelDesc d = desc(a);
    if (l == 0 && with_dots && tiled_dots(a) && nu_post_ == 2) {
      dim3 grid((a.mx + TX - 1) / TX, (a.my + TY - 1) / TY);
      const FcgDotsIn fd{r64_.get(), p_[0].get(), q_.get(), acc_.get(), L_.Cx, L_.Cy, L_.Cd};
      launch_pdl(k_smooth_tile<false, true>, grid, dim3(kSmoothThreads), 0, s, a.u.get(), a.u2.get(), a.f.get(), d, result(l + 1), desc(b), st, nullptr, fd);
      a.result_in_u2 = true;
      fused_dots = true;
    } else if (tiled(a) && nu_post_ == 2) {
      dim3 grid((a.mx + TX - 1) / TX, (a.my + TY - 1) / TY);
      launch_pdl(k_smooth_tile<false>, grid, dim3(kSmoothThreads), 0, s, a.u.get(), a.u2.get(), a.f.get(), d, result(l + 1), desc(b), st, nullptr, FcgDotsIn{});
      a.result_in_u2 = true;
    } else {
      a.result_in_u2 = false;
      launch_pdl(k_prolong_generic, dim3(blocks_for(a.mx * a.my)), dim3(256), 0, s, result(l + 1), desc(b), a.u.get(), d, st);
      for (int it = 0; it < nu_post_; ++it) {
        launch_pdl(k_smooth_generic, dim3(blocks_for((a.mx + 1) / 2 * a.my)), dim3(256), 0, s, a.u.get(), a.f.get(), d, 1, st);
        launch_pdl(k_smooth_generic, dim3(blocks_for((a.mx + 1) / 2 * a.my)), dim3(256), 0, s, a.u.get(), a.f.get(), d, 0, st);
      }
    }
  }
  return fused_dots;
}

// One FCG iteration (parity: which direction buffer is current).
void PoissonMG::enqueue_iteration(int parity, double* x, double tol, int maxiter, cudaStream_t s) {
  double* st = state_.get();
  Level& f = lv_[0];
  const double wsum = singular_ ? wsum_ : double(n_);
  if (singular_) {
    launch_pdl(k_sub_mean32, dim3(blocks_for(n_)), dim3(256), 0, s, f.f.get(), n_, st);
  }
  const bool fused = vcycle(s, true);  // z = M r (and pass A, when fused)
  const float* z = result(0);
  (void)parity;  // p and q are updated in place
  if (!fused) {
    launch_pdl(k_fcg_dots, dim3(reduce_blocks(n_)), dim3(256), 0, s, z, q_.get(), p_[0].get(), r64_.get(), L_, st, acc_.get());
  }
  launch_pdl(k_fcg_step, dim3((n_ + kStepThreads * kStepPoints - 1) / (kStepThreads * kStepPoints)),
             dim3(kStepThreads), 0, s, z, p_[0].get(), q_.get(), x, r64_.get(),
             f.f.get(), L_, st, acc_.get(), ctr_.get(), tol, maxiter, wsum);
  GP_LAUNCH_CHECK();
}

// The two iteration graphs (even and odd parity) for this solution vector
// and stopping rule, captured on first use in thread-local mode (other host
// threads driving other simulations are not affected). Kernel launches are
// counted when a graph is launched, not when it is captured. An empty result
// (exec[0] == nullptr) means direct launches: the stream is already being
// captured by the caller, or the capture failed.
PoissonMG::IterationGraphs PoissonMG::iteration_graphs(double* x, double tol, int maxiter, cudaStream_t s) {
  for (const auto& g : graphs_)
    if (g.x == x && g.tol == tol && g.maxiter == maxiter) return g;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (!graphs_ok_ || cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone)
    return IterationGraphs{};
  IterationGraphs g{};
  g.x = x;
  g.tol = tol;
  g.maxiter = maxiter;
  const unsigned long long c0 = thread_kernel_launches();
  bool ok = true;
  for (int par = 0; par < 1 && ok; ++par) {  // one graph: p and q are updated in place
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      ok = false;
      break;
    }
    try {
      enqueue_iteration(par, x, tol, maxiter, s);
    } catch (...) {
      ok = false;
    }
    if (cudaStreamEndCapture(s, &graph) != cudaSuccess || !graph) ok = false;
    if (ok && cudaGraphInstantiate(&g.exec[par], graph, 0) != cudaSuccess) ok = false;
    if (graph) cudaGraphDestroy(graph);
  }
  const unsigned long long captured = thread_kernel_launches() - c0;
  add_kernel_launches(-static_cast<long long>(captured));
  (void)cudaGetLastError();
  if (!ok) {
    for (auto& e : g.exec)
      if (e) cudaGraphExecDestroy(e);
    graphs_ok_ = false;
    return IterationGraphs{};
  }
  g.kernels = static_cast<long long>(captured);
  if (graphs_.size() >= 4) {  // a few solution vectors per system (Poisson, Darwin parts, tests)
    for (auto& e : graphs_.front().exec) cudaGraphExecDestroy(e);
    graphs_.erase(graphs_.begin());
  }
  graphs_.push_back(g);
  return g;
}

PoissonMG::~PoissonMG() {
  for (auto& g : graphs_)
    for (auto& e : g.exec)
      if (e) cudaGraphExecDestroy(e);
}

MGResult PoissonMG::solve(const double* b, const double* sums_b, double* x, double tol, int maxiter,
                          cudaStream_t s) {
  MGResult res;
  double* st = state_.get();
  Level& f = lv_[0];
  const bool singular = singular_;
  launch_pdl(k_init, dim3(blocks_for(n_)), dim3(256), 0, s, st, sums_b, acc_.get(), x, n_);
  const double wsum = singular_ ? wsum_ : double(n_);
  launch_pdl(k_residual64, dim3(reduce_blocks(n_)), dim3(256), 0, s, x, b, L_, f.f.get(), r64_.get(), st,
             ctr_.get(), tol, maxiter, wsum);
  // Batches of iterations without host synchronisation; every kernel returns
  // at once after convergence. The batch size follows the last solve. An
  // iteration is one CUDA graph launch when its graph could be captured.
  const IterationGraphs gr = iteration_graphs(x, tol, maxiter, s);
  int batch = last_iters_ > 0 ? last_iters_ : 1;
  int launched = 0;
  for (;;) {
    for (int i = 0; i < batch && launched < maxiter; ++i, ++launched) {
      if (gr.exec[0]) {
        GP_CUDA(cudaGraphLaunch(gr.exec[0], s));
        add_kernel_launches(gr.kernels);
      } else {
        enqueue_iteration(launched & 1, x, tol, maxiter, s);
      }
    }
    GP_CUDA(cudaMemcpyAsync(host_.get(), st, S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, s));
    GP_CUDA(cudaStreamSynchronize(s));
    if (host_[S_DONE] != 0.0 || launched >= maxiter) break;
    batch = 1;
  }
  res.norm_b = host_[S_NORMB];
  res.rel_residual = host_[S_REL];
  res.rel0 = host_[S_REL0];
  res.iterations = int(host_[S_ITER]);
  if (host_[S_DONE] == 2.0) {
    res.iterations = 0;
    return res;
  }
  last_iters_ = res.iterations > 0 ? res.iterations : 1;
  if (singular) {  // gauge: zero-mean solution
    GP_CUDA(cudaMemsetAsync(st + S_SUM, 0, sizeof(double), s));
    k_sum64<<<blocks_for(n_), 256, 0, s>>>(x, n_, st + S_SUM);
    GP_LAUNCH_CHECK();
    k_sub_mean64<<<blocks_for(n_), 256, 0, s>>>(x, n_, st + S_SUM);
    GP_LAUNCH_CHECK();
  }
  return res;
}

}  // namespace gample
