// sort_kernels.cu -- counting sort of the particles by cell (sm_100a).
//
// Key: the particle's cell in tile-major order (8 x 8-cell tiles, row-major
// over tiles, row-major inside a tile), so consecutive particles share a cell
// and a chunk of consecutive particles covers a compact box. Three passes:
// histogram (warp-aggregated atomics: lanes with equal keys add once),
// exclusive scan of the counts, scatter into the spare buffer (slots claimed
// with warp-aggregated atomics). The order inside a cell is unspecified.
#include <cuda_runtime.h>

#include "device.hpp"
#include "kernels.hpp"
#include "pic_common.cuh"

namespace gample {
namespace kern {

namespace {

constexpr int kTile = 8;
constexpr int kThreads = 256;
constexpr int kScanThreads = 1024;
constexpr int kScanPer = 4;
constexpr int kScanChunk = kScanThreads * kScanPer;
constexpr unsigned kNoKey = 0xffffffffu;

struct KeyGeom {
  int ntx;       // tiles per row
  uint32_t nkeys;
};

__device__ __forceinline__ uint32_t cell_key(int32_t cell, const KeyGeom& k) {
  if (cell < 0) return k.nkeys;  // flagged particles (none after compaction) go last
  const int ix = cell_ix(cell), iy = cell_iy(cell);
  const uint32_t tile = uint32_t((iy / kTile) * k.ntx + ix / kTile);
  return (tile * kTile + uint32_t(iy % kTile)) * kTile + uint32_t(ix % kTile);
}

__global__ void __launch_bounds__(kThreads) k_cs_hist(const int32_t* cell, const SpeciesCounters* cnt, KeyGeom g,
                                                      uint32_t* counts) {
  const uint32_t n = cnt->n;
  const int lane = threadIdx.x & 31;
  for (uint32_t base = (blockIdx.x * kThreads + threadIdx.x) & ~31u; base < n; base += gridDim.x * kThreads) {
    const uint32_t k = base + lane;
    const uint32_t key = k < n ? cell_key(cell[k], g) : kNoKey;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    if (key != kNoKey && lane == __ffs(peers) - 1) atomicAdd(&counts[key], uint32_t(__popc(peers)));
  }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_local(const uint32_t* in, uint32_t* out, uint32_t* sums,
                                                             uint32_t n) {
  __shared__ uint32_t s_warp[32];
  const uint32_t base = blockIdx.x * uint32_t(kScanChunk) + threadIdx.x * kScanPer;
  uint32_t v[kScanPer], t = 0;
#pragma unroll
  for (int i = 0; i < kScanPer; ++i) {
    v[i] = base + i < n ? in[base + i] : 0u;
    t += v[i];
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t incl = t;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) s_warp[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    const uint32_t x = s_warp[lane];
    uint32_t xi = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, xi, o);
      if (lane >= o) xi += y;
    }
    s_warp[lane] = xi - x;
    if (lane == 31) sums[blockIdx.x] = xi;
  }
  __syncthreads();
  uint32_t run = s_warp[wid] + incl - t;
#pragma unroll
  for (int i = 0; i < kScanPer; ++i) {
    if (base + i < n) out[base + i] = run;
    run += v[i];
  }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_sums(uint32_t* sums, uint32_t nb) {
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_base;
  if (threadIdx.x == 0) s_base = 0;
  __syncthreads();
  for (uint32_t b0 = 0; b0 < nb; b0 += kScanThreads) {
    const uint32_t b = b0 + threadIdx.x;
    const uint32_t c = b < nb ? sums[b] : 0u;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      const uint32_t x = s_warp[lane];
      uint32_t xi = x;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, xi, o);
        if (lane >= o) xi += y;
      }
      s_warp[lane] = xi - x;
    }
    __syncthreads();
    if (b < nb) sums[b] = s_base + s_warp[wid] + incl - c;
    __syncthreads();
    if (threadIdx.x == kScanThreads - 1) s_base += s_warp[wid] + incl;
    __syncthreads();
  }
}

__global__ void k_scan_add(uint32_t* out, const uint32_t* sums, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += sums[i / kScanChunk];
}

__global__ void __launch_bounds__(kThreads) k_cs_scatter(ParticleArrays src, ParticleArrays dst,
                                                         const SpeciesCounters* cnt, KeyGeom g, uint32_t* offsets) {
  const uint32_t n = cnt->n;
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  for (uint32_t base = (blockIdx.x * kThreads + threadIdx.x) & ~31u; base < n; base += gridDim.x * kThreads) {
    const uint32_t k = base + lane;
    const uint32_t key = k < n ? cell_key(src.cell[k], g) : kNoKey;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int leader = __ffs(peers) - 1;
    uint32_t slot = 0;
    if (key != kNoKey && lane == leader) slot = atomicAdd(&offsets[key], uint32_t(__popc(peers)));
    slot = __shfl_sync(0xffffffffu, slot, leader) + uint32_t(__popc(peers & lt));
    if (key != kNoKey) {
      dst.cell[slot] = src.cell[k];
      dst.ox[slot] = src.ox[k];
      dst.oy[slot] = src.oy[k];
      dst.vx[slot] = src.vx[k];
      dst.vy[slot] = src.vy[k];
      dst.vz[slot] = src.vz[k];
    }
  }
}

KeyGeom geom(GridDims g) {
  KeyGeom k;
  k.ntx = (g.nx + kTile) / kTile;
  const int nty = (g.ny + kTile) / kTile;
  k.nkeys = uint32_t(k.ntx) * uint32_t(nty) * kTile * kTile;
  return k;
}

int grid_for(uint32_t n) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    GP_CUDA(cudaGetDevice(&dev));
    GP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  }
  long long need = ((long long)n + kThreads - 1) / kThreads;
  long long cap = (long long)sms * 8;
  if (need < 1) need = 1;
  return int(need < cap ? need : cap);
}

}  // namespace

size_t sort_key_count(GridDims g) { return size_t(geom(g).nkeys) + 1; }

size_t sort_scratch_words(GridDims g) {
  const size_t nk = sort_key_count(g);
  return 2 * nk + (nk + kScanChunk - 1) / kScanChunk + 32;
}

void sort_by_cell(GridDims g, ParticleArrays src, ParticleArrays dst, const SpeciesCounters* cnt, uint32_t* scratch,
                  uint32_t n_bound, cudaStream_t s) {
  if (n_bound == 0) return;
  const KeyGeom kg = geom(g);
  const uint32_t nk = kg.nkeys + 1;
  uint32_t* counts = scratch;
  uint32_t* offsets = scratch + nk;
  uint32_t* sums = scratch + 2 * size_t(nk);
  const uint32_t nb = (nk + kScanChunk - 1) / kScanChunk;
  GP_CUDA(cudaMemsetAsync(counts, 0, size_t(nk) * sizeof(uint32_t), s));
  k_cs_hist<<<grid_for(n_bound), kThreads, 0, s>>>(src.cell, cnt, kg, counts);
  GP_LAUNCH_CHECK();
  k_scan_local<<<nb, kScanThreads, 0, s>>>(counts, offsets, sums, nk);
  GP_LAUNCH_CHECK();
  k_scan_sums<<<1, kScanThreads, 0, s>>>(sums, nb);
  GP_LAUNCH_CHECK();
  k_scan_add<<<(nk + 255) / 256, 256, 0, s>>>(offsets, sums, nk);
  GP_LAUNCH_CHECK();
  k_cs_scatter<<<grid_for(n_bound), kThreads, 0, s>>>(src, dst, cnt, kg, offsets);
  GP_LAUNCH_CHECK();
}

}  // namespace kern
}  // namespace gample
