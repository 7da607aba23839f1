// darwin_kernels.cu -- right-hand sides and field corrections of the Darwin
// model (src/EMField.mm:1138-1361) on the vector-potential grid of
// (nkx+1)(nky+1) nodes (src/EMField.mm:484-492): nkx = ngx, minus one when x
// is periodic (same in y); node (i, j) sits at rho index (i+ngb, j+ngb).
#include <cuda_runtime.h>

#include "device.hpp"
#include "kernels.hpp"

namespace gample {
namespace kern {

namespace {

constexpr double kPI = 3.141592653589793;
constexpr double kC = 2.99792458e10;

__device__ __forceinline__ double block_sum2(double v, double* sh) {
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

int grid_for(int n) {
  const int b = (n + 255) / 256;
  return b < 1 ? 1 : (b < 1184 ? b : 1184);
}

// div J with the Neumann boundary terms (src/EMField.mm:1150-1184), FP32
// differences as the reference evaluates them, accumulated in FP64.
__global__ void k_div_rhs(const float* jx, const float* jy, DarwinGeom G, double* rhs) {
  const int mx = G.nkx + 1, n = mx * (G.nky + 1);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int i = k % mx, j = k / mx;
    const int ix = i + G.ngb, jy0 = j + G.ngb;
    double r = 0.0;
    if (!G.perx) {
      if (i == 0)
        r += double(__fdiv_rn(-2.0f * jx[ix + jy0 * (G.nx + 2)], G.dx));
      else if (i == G.nkx)
        r += double(__fdiv_rn(2.0f * jx[ix + jy0 * (G.nx + 2)], G.dx));
    }
    if (!G.pery) {
      if (j == 0)
        r += double(__fdiv_rn(-2.0f * jy[ix + jy0 * (G.nx + 1)], G.dy));
      else if (j == G.nky)
        r += double(__fdiv_rn(2.0f * jy[ix + jy0 * (G.nx + 1)], G.dy));
    }
    const double djx = double(__fdiv_rn(__fsub_rn(jx[ix + 1 + jy0 * (G.nx + 2)], jx[ix + jy0 * (G.nx + 2)]), G.dx));
    const double djy = double(__fdiv_rn(__fsub_rn(jy[ix + (jy0 + 1) * (G.nx + 1)], jy[ix + jy0 * (G.nx + 1)]), G.dy));
    rhs[k] = r + (djx + djy);
  }
}

// -(4 pi / c) (J_a - d_a psi) on the J_a nodes (src/EMField.mm:1201-1275);
// dir 0: x, 1: y. The last column (row) is 0 in the reference; with a
// periodic direction the build closes it through the wrap.
__global__ void k_a_rhs(const float* ja, const double* psi, DarwinGeom G, int dir, double* rhs) {
  const int mx = G.nkx + 1, n = mx * (G.nky + 1);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int i = k % mx, j = k / mx;
    double r = 0.0;
    if (dir == 0) {
      if (i < G.nkx || G.perx) {
        const int k1 = i < G.nkx ? k + 1 : k - G.nkx;
        const double jl = (psi[k1] - psi[k]) / double(G.dx);
        r = -4 * kPI / kC * (double(ja[(i + G.ngb + 1) + (j + G.ngb) * (G.nx + 2)]) - jl);
      }
    } else {
      if (j < G.nky || G.pery) {
        const int k1 = j < G.nky ? k + mx : k - G.nky * mx;
        const double jl = (psi[k1] - psi[k]) / double(G.dy);
        r = -4 * kPI / kC * (double(ja[(i + G.ngb) + (j + G.ngb + 1) * (G.nx + 1)]) - jl);
      }
    }
    rhs[k] = r;
  }
}

// v -= (sum w v) / (sum w) with the solvability weights (1/2 at Neumann ends).
__global__ void k_wsum(const double* v, DarwinGeom G, double* out) {
  __shared__ double sh[32];
  const int mx = G.nkx + 1, my = G.nky + 1, n = mx * my;
  double s = 0.0, w = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int i = k % mx, j = k / mx;
    const double wi = (!G.perx && (i == 0 || i == mx - 1)) ? 0.5 : 1.0;
    const double wj = (!G.pery && (j == 0 || j == my - 1)) ? 0.5 : 1.0;
    s += wi * wj * v[k];
    w += wi * wj;
  }
  s = block_sum2(s, sh);
  w = block_sum2(w, sh);
  if (threadIdx.x == 0) {
    atomicAdd(out, s);
    atomicAdd(out + 1, w);
  }
}

__global__ void k_wsub(double* v, int n, const double* sw) {
  const double m = sw[0] / sw[1];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) v[k] -= m;
}

// delE = -(A - A_last) / (c dt), delBz = d_x Ay - d_y Ax (src/EMField.mm:1277-1297)
// at the J nodes; A_last <- A.
__global__ void k_fields(const double* Ax, const double* Ay, const double* lastAx, const double* lastAy, DarwinGeom G,
                         double cdt, float* delEx, float* delEy, float* delBz) {
  const int mx = G.nkx + 1;
  const int ni = G.perx ? G.nkx + 1 : G.nkx, nj = G.pery ? G.nky + 1 : G.nky;
  const int n = ni * nj;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int i = t % ni, j = t / ni;
    const int kf = i + j * mx;
    const int kx1 = i < G.nkx ? kf + 1 : kf - G.nkx;          // i + 1 (wrapped when periodic)
    const int ky1 = j < G.nky ? kf + mx : kf - G.nky * mx;    // j + 1
    const int kpx = (i + G.ngb + 1) + (j + G.ngb) * (G.nx + 2);
    const int kpy = (i + G.ngb) + (j + G.ngb + 1) * (G.nx + 1);
    delEx[kpx] = float(-(Ax[kf] - lastAx[kf]) / cdt);
    delEy[kpy] = float(-(Ay[kf] - lastAy[kf]) / cdt);
    const double dyAx = (Ax[ky1] - Ax[kf]) / double(G.dy);
    const double dxAy = (Ay[kx1] - Ay[kf]) / double(G.dx);
    delBz[kpx + (G.nx + 2)] = float(dxAy - dyAx);
  }
}

}  // namespace

void darwin_div_rhs(const float* jx, const float* jy, DarwinGeom G, double* rhs, cudaStream_t s) {
  const int n = (G.nkx + 1) * (G.nky + 1);
  k_div_rhs<<<grid_for(n), 256, 0, s>>>(jx, jy, G, rhs);
  GP_LAUNCH_CHECK();
}

void darwin_a_rhs(const float* ja, const double* psi, DarwinGeom G, int dir, double* rhs, cudaStream_t s) {
  const int n = (G.nkx + 1) * (G.nky + 1);
  k_a_rhs<<<grid_for(n), 256, 0, s>>>(ja, psi, G, dir, rhs);
  GP_LAUNCH_CHECK();
}

void darwin_weighted_project(double* v, DarwinGeom G, double* scratch2, cudaStream_t s) {
  const int n = (G.nkx + 1) * (G.nky + 1);
  GP_CUDA(cudaMemsetAsync(scratch2, 0, 2 * sizeof(double), s));
  k_wsum<<<grid_for(n), 256, 0, s>>>(v, G, scratch2);
  GP_LAUNCH_CHECK();
  k_wsub<<<grid_for(n), 256, 0, s>>>(v, n, scratch2);
  GP_LAUNCH_CHECK();
}

void darwin_fields(const double* Ax, const double* Ay, const double* lastAx, const double* lastAy, DarwinGeom G,
                   double cdt, float* delEx, float* delEy, float* delBz, cudaStream_t s) {
  const int n = (G.nkx + 1) * (G.nky + 1);
  k_fields<<<grid_for(n), 256, 0, s>>>(Ax, Ay, lastAx, lastAy, G, cdt, delEx, delEy, delBz);
  GP_LAUNCH_CHECK();
}

}  // namespace kern
}  // namespace gample
