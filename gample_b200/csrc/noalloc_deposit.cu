// noalloc_deposit.cu -- charge deposit into caller-owned device memory that
// allocates nothing (the gp_deposit_charge_noalloc entry point).
//
// For callers that already own every device buffer and may not let a library
// allocate: a host framework running a fixed device-memory budget or its own
// pool, or a time loop that must not pay the implicit device synchronisation
// of cudaMalloc / cudaFree. The particles are the reference's 24-byte records
// (src/Particle.h:14-21) already in device memory; the result is the charge
// density of one species in the reference's rho layout, (nx+1)(ny+1) floats
// (src/EMField.mm:127-144), computed like the deterministic deposit of the
// handle API: weights quantised to 2^-40, exact int64 sums, one rounding to
// float at the end.
//
// Scratch: the int64 accumulator lives in a file-scope __device__ array of
// kMaxNodes entries (8 MiB), so grids with (nx+1)(ny+1) > kMaxNodes are
// rejected. Its device address is looked up with cudaGetSymbolAddress on every
// call, in the caller's current context (a lookup, not an allocation): an
// address kept from an earlier call would be stale after cudaDeviceReset or
// in another context on the same device. The first call on a device may load
// this library's device code, so it should come before any stream capture.
// Every call clears the part it uses before depositing (cudaMemsetAsync, no
// allocation), so nothing has to start at zero; rho is overwritten. All calls
// on one device share the array: calls that overlap in time (different
// streams or host threads without ordering between them) race and corrupt
// each other's results.
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "device.hpp"
#include "kernels.hpp"
#include "pic_common.cuh"

namespace gample {
namespace kern {

namespace {

constexpr size_t kMaxNodes = size_t(1) << 20;
constexpr int kBlock = 256;

static __device__ __align__(256) unsigned long long g_noalloc_acc[kMaxNodes];

// Deterministic fixed-point deposit of one particle record per thread; the
// record is split into cell and offset as the handle API's upload does, and
// the weights are the same Horner-form B-splines (src/Particle.mm:311-373).
template <int ORDER>
__global__ void k_deposit_records(const ParticleStateAoS* in, uint32_t n, GridDims g, unsigned long long* acc) {
  const int nx = g.nx, ny = g.ny, ngb = g.ngb;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const ParticleStateAoS r = in[k];
    const float fx = floorf(r.x), fy = floorf(r.y);
    const int ix = int(fx), iy = int(fy);
    const bool ok = isfinite(r.x) && isfinite(r.y) && ix >= 0 && iy >= 0 && ix < 65536 && iy < 32768;
    if (r.piflag != 0 || !ok) continue;
    const Stagger sx = stagger(ix, __fsub_rn(r.x, fx)), sy = stagger(iy, __fsub_rn(r.y, fy));
    float wx[ORDER + 1], wy[ORDER + 1];
    shape<ORDER>(sx.hnode, wx);
    shape<ORDER>(sy.hnode, wy);
    const int rc = sx.node - ngb, rr = sy.node - ngb;
#pragma unroll
    for (int i = 0; i <= ORDER; ++i)
#pragma unroll
      for (int j = 0; j <= ORDER; ++j) {
        const int col = rc + i, row = rr + j;
        if (col < 0 || row < 0 || col > nx || row > ny) continue;
        atomicAdd(acc + col + size_t(row) * (nx + 1),
                  static_cast<unsigned long long>(quant40(__fmul_rn(wx[i], wy[j]))));
      }
  }
}

__global__ void k_round_records(const unsigned long long* acc, size_t n, double f, float* rho) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    rho[i] = __double2float_rn(__dadd_rn(0.0, __dmul_rn(double(static_cast<long long>(acc[i])), f)));
}

unsigned long long* scratch_address() {
  void* p = nullptr;
  const cudaError_t rc = cudaGetSymbolAddress(&p, g_noalloc_acc);
  if (rc != cudaSuccess || !p)
    throw CudaError(rc, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(rc));
  return static_cast<unsigned long long*>(p);
}

int blocks_for(size_t work) {
  const size_t b = (work + kBlock - 1) / kBlock;
  return int(b < 148 * 16 ? (b ? b : 1) : 148 * 16);
}

}  // namespace

size_t noalloc_max_nodes() { return kMaxNodes; }

void deposit_charge_noalloc(int order, int ngx, int ngy, const ParticleStateAoS* particles, uint32_t n, float scale,
                            float* rho, cudaStream_t s) {
  if (order != 1 && order != 3 && order != 5) throw std::invalid_argument("weighting order must be 1, 3 or 5");
  if (ngx < 1 || ngy < 1 || ngx > 65000 || ngy > 32000) throw std::invalid_argument("grid size out of range");
  if (!rho || (n && !particles)) throw std::invalid_argument("null device pointer");
  GridDims g;
  g.ngx = ngx;
  g.ngy = ngy;
  g.ngb = order / 2;
  g.nx = ngx + 2 * g.ngb;
  g.ny = ngy + 2 * g.ngb;
  const size_t nodes = size_t(g.nx + 1) * size_t(g.ny + 1);
  if (nodes > kMaxNodes)
    throw std::length_error("grid needs " + std::to_string(nodes) + " rho nodes; the allocation-free deposit holds " +
                            std::to_string(kMaxNodes));
  unsigned long long* acc = scratch_address();
  GP_CUDA(cudaMemsetAsync(acc, 0, nodes * sizeof(unsigned long long), s));
  if (n) {
    switch (order) {
      case 1: k_deposit_records<1><<<blocks_for(n), kBlock, 0, s>>>(particles, n, g, acc); break;
      case 3: k_deposit_records<3><<<blocks_for(n), kBlock, 0, s>>>(particles, n, g, acc); break;
      default: k_deposit_records<5><<<blocks_for(n), kBlock, 0, s>>>(particles, n, g, acc); break;
    }
    GP_LAUNCH_CHECK();
  }
  // same factor and rounding as the handle API's combine of one species
  const double f = double(scale) * 0x1p-40 * 1.0;
  k_round_records<<<blocks_for(nodes), kBlock, 0, s>>>(acc, nodes, f, rho);
  GP_LAUNCH_CHECK();
}

}  // namespace kern
}  // namespace gample
