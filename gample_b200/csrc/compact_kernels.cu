// compact_kernels.cu -- particle compaction and record conversion (sm_100a).
//
// Compaction removes the particles flagged by the push (dead bitmap) and
// fills each hole, in ascending order, with the last live particle, in
// descending order -- the permutation of the reference's serial loop
// (src/Particle.mm:893-966), computed with prefix sums over the bitmap.
#include <cuda_runtime.h>

#include "device.hpp"
#include "pdl.cuh"
#include "kernels.hpp"
#include "pic_common.cuh"

namespace gample {
namespace kern {

namespace {

constexpr int kBlock = 256;

int grid_for(uint32_t n_bound) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    GP_CUDA(cudaGetDevice(&dev));
    GP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  }
  long long need = ((long long)n_bound + kBlock - 1) / kBlock;
  long long cap = (long long)sms * 8;
  if (need < 1) need = 1;
  return int(need < cap ? need : cap);
}
// ---------------------------------------------------------- compaction
// scratch layout (uint32 words):
//   [0] n_live   [1] tail count   [2..15] reserved
//   [16, 16 + kMaxScanBlocks)      per-block hole counts (exclusive-scanned in place)
//   [16 + kMaxScanBlocks, ...)     tail list (live indices >= n_live, descending)
constexpr int kWordsPerThread = 8;
constexpr int kHoleBlock = 256;
constexpr uint32_t kWordsPerBlock = kWordsPerThread * kHoleBlock;  // 2048 words = 65536 particles
constexpr uint32_t kMaxScanBlocks = 65536;                       // up to 2^32 particles

__device__ __forceinline__ uint32_t live_mask_range(uint32_t w, uint32_t lo, uint32_t hi) {
  // bits of word w whose particle index is in [lo, hi)
  const uint32_t b0 = w * 32u;
  uint32_t m = 0xffffffffu;
  if (lo > b0) m &= (lo - b0 >= 32u) ? 0u : (0xffffffffu << (lo - b0));
  if (hi < b0 + 32u) m &= (hi <= b0) ? 0u : (0xffffffffu >> (32u - (hi - b0)));
  return m;
}

// One block: list the live particles in [n_live, n) from the top down and
// publish n_live; the counters' n becomes n_live.
__global__ void __launch_bounds__(1024) k_compact_tail(SpeciesCounters* cnt, const uint32_t* bits,
                                                       uint32_t* scratch) {
  grid_dependency_wait();
  grid_dependents_launch();
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_base;
  const uint32_t n = cnt->n, nd = cnt->n_dead;
  const uint32_t nl = n - nd;
  if (threadIdx.x == 0) s_base = 0;
  __syncthreads();
  uint32_t* tail = scratch + 16 + kMaxScanBlocks;
  if (nd > 0) {
    const int w_hi = int((n - 1) >> 5), w_lo = int(nl >> 5);
    for (int w0 = w_hi; w0 >= w_lo; w0 -= int(blockDim.x)) {
      const int w = w0 - int(threadIdx.x);
      uint32_t live = 0;
      if (w >= w_lo) live = ~bits[w] & live_mask_range(uint32_t(w), nl, n);
      const uint32_t c = __popc(live);
      // block exclusive scan of c
      const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
      uint32_t incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      if (lane == 31) s_warp[wid] = incl;
      __syncthreads();
      if (wid == 0) {
        uint32_t v = s_warp[lane];
        uint32_t vi = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          uint32_t t = __shfl_up_sync(0xffffffffu, vi, o);
          if (lane >= o) vi += t;
        }
        s_warp[lane] = vi - v;
      }
      __syncthreads();
      uint32_t pos = s_base + s_warp[wid] + incl - c;
      for (int b = 31; b >= 0; --b)
        if (live >> b & 1u) tail[pos++] = uint32_t(w) * 32u + uint32_t(b);
      __syncthreads();
      if (threadIdx.x == blockDim.x - 1) s_base += s_warp[wid] + incl;
      __syncthreads();
    }
  }
  if (threadIdx.x == 0) {
    scratch[0] = nl;
    scratch[1] = s_base;
    cnt->n = nl;
    cnt->n_pulled = nd;
    cnt->n_dead = 0;  // consumed: a second compaction without a push is a no-op
  }
}

// nw_bound: words below the host's bound of the count (in bounds); they are
// read while n_live is still being loaded, then masked with it.
__global__ void __launch_bounds__(kHoleBlock) k_hole_count(const uint32_t* bits, uint32_t* scratch,
                                                           uint32_t nw_bound) {
  grid_dependency_wait();
  grid_dependents_launch();
  __shared__ uint32_t s_red[kHoleBlock / 32];
  const uint32_t nl = scratch[0];
  const uint32_t w0 = blockIdx.x * kWordsPerBlock + threadIdx.x * kWordsPerThread;
  uint32_t raw[kWordsPerThread];
#pragma unroll
  for (int t = 0; t < kWordsPerThread; ++t) raw[t] = w0 + t < nw_bound ? bits[w0 + t] : 0u;
  uint32_t c = 0;
#pragma unroll
  for (int t = 0; t < kWordsPerThread; ++t) c += __popc(raw[t] & live_mask_range(w0 + t, 0, nl));
  c = __reduce_add_sync(0xffffffffu, c);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t s = 0;
    for (int i = 0; i < kHoleBlock / 32; ++i) s += s_red[i];
    scratch[16 + blockIdx.x] = s;
  }
}

__global__ void __launch_bounds__(1024) k_scan_blocks(uint32_t* scratch, uint32_t nblocks) {
  grid_dependency_wait();
  grid_dependents_launch();
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_base;
  if (threadIdx.x == 0) s_base = 0;
  __syncthreads();
  uint32_t* v = scratch + 16;
  for (uint32_t b0 = 0; b0 < nblocks; b0 += blockDim.x) {
    const uint32_t b = b0 + threadIdx.x;
    const uint32_t c = b < nblocks ? v[b] : 0u;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      uint32_t x = s_warp[lane], xi = x;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, xi, o);
        if (lane >= o) xi += t;
      }
      s_warp[lane] = xi - x;
    }
    __syncthreads();
    if (b < nblocks) v[b] = s_base + s_warp[wid] + incl - c;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) s_base += s_warp[wid] + incl;
    __syncthreads();
  }
}

// As k_hole_count, the bit words and this block's first rank are read
// together with n_live.
__global__ void __launch_bounds__(kHoleBlock) k_fill_holes(ParticleArrays p, const uint32_t* bits,
                                                           const uint32_t* scratch, uint32_t nw_bound) {
  grid_dependency_wait();
  grid_dependents_launch();
  __shared__ uint32_t s_warp[kHoleBlock / 32];
  const uint32_t nl = scratch[0];
  const uint32_t block_rank = scratch[16 + blockIdx.x];
  const uint32_t w0 = blockIdx.x * kWordsPerBlock + threadIdx.x * kWordsPerThread;
  uint32_t m[kWordsPerThread];
#pragma unroll
  for (int t = 0; t < kWordsPerThread; ++t) m[t] = w0 + t < nw_bound ? bits[w0 + t] : 0u;
  uint32_t c = 0;
#pragma unroll
  for (int t = 0; t < kWordsPerThread; ++t) {
    m[t] &= live_mask_range(w0 + t, 0, nl);
    c += __popc(m[t]);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) s_warp[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    uint32_t x = lane < kHoleBlock / 32 ? s_warp[lane] : 0u, xi = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(0xffffffffu, xi, o);
      if (lane >= o) xi += t;
    }
    if (lane < kHoleBlock / 32) s_warp[lane] = xi - x;
  }
  __syncthreads();
  uint32_t rank = block_rank + s_warp[wid] + incl - c;
  const uint32_t* tail = scratch + 16 + kMaxScanBlocks;
#pragma unroll
  for (int t = 0; t < kWordsPerThread; ++t) {
    uint32_t mm = m[t];
    while (mm) {
      const int b = __ffs(mm) - 1;
      mm &= mm - 1;
      const uint32_t dst = (w0 + t) * 32u + uint32_t(b);
      const uint32_t src = tail[rank++];
      p.cell[dst] = p.cell[src];
      p.ox[dst] = p.ox[src];
      p.oy[dst] = p.oy[src];
      p.vx[dst] = p.vx[src];
      p.vy[dst] = p.vy[src];
      p.vz[dst] = p.vz[src];
    }
  }
}

// A record is kept live only if its cell lies within the field arrays
// (0 <= ix <= nx, 0 <= iy <= ny): the cell sort's keys and every stencil
// start from there. Anything else, or a non-finite position, is an invalid state.
__global__ void k_aos_to_soa(const ParticleStateAoS* in, uint32_t n, ParticleArrays p, int nx, int ny) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const ParticleStateAoS r = in[k];
    const bool fin = isfinite(r.x) && isfinite(r.y) && fabsf(r.x) < 1.0e7f && fabsf(r.y) < 1.0e7f;
    const float fx = fin ? floorf(r.x) : 0.0f, fy = fin ? floorf(r.y) : 0.0f;
    int ix = int(fx), iy = int(fy);
    bool ok = fin && ix >= 0 && iy >= 0 && ix <= nx && iy <= ny;
    if (r.piflag != 0 || !ok) {  // a wall code 1..4 is kept; anything else is an invalid state
      p.cell[k] = -(r.piflag >= 1 && r.piflag <= 4 ? r.piflag : 5);
      p.ox[k] = 0.0f;
      p.oy[k] = 0.0f;
    } else {
      p.cell[k] = pack_cell(ix, iy);
      p.ox[k] = __fsub_rn(r.x, fx);
      p.oy[k] = __fsub_rn(r.y, fy);
    }
    p.vx[k] = r.vx;
    p.vy[k] = r.vy;
    p.vz[k] = r.vz;
  }
}

__global__ void k_soa_to_aos(ParticleArrays p, uint32_t n, ParticleStateAoS* out) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    ParticleStateAoS r;
    const int32_t c = p.cell[k];
    if (c >= 0) {
      r.x = __fadd_rn(float(cell_ix(c)), p.ox[k]);
      r.y = __fadd_rn(float(cell_iy(c)), p.oy[k]);
      r.piflag = 0;
    } else {
      r.x = __int_as_float(0x7fc00000);
      r.y = r.x;
      r.piflag = -c;
    }
    r.vx = p.vx[k];
    r.vy = p.vy[k];
    r.vz = p.vz[k];
    out[k] = r;
  }
}

}  // namespace

size_t compact_scratch_words(uint32_t n_bound) { return 16 + size_t(kMaxScanBlocks) + size_t(n_bound) + 32; }

void compact(ParticleArrays p, SpeciesCounters* cnt, const uint32_t* dead_bits, uint32_t* scratch,
             uint32_t n_bound, cudaStream_t s) {
  if (n_bound == 0) return;
  launch_pdl(k_compact_tail, dim3(1), dim3(1024), 0, s, cnt, dead_bits, scratch);
  const uint32_t nwords = (n_bound + 31u) / 32u;
  const uint32_t nblocks = (nwords + kWordsPerBlock - 1) / kWordsPerBlock;
  launch_pdl(k_hole_count, dim3(nblocks), dim3(kHoleBlock), 0, s, dead_bits, scratch, nwords);
  launch_pdl(k_scan_blocks, dim3(1), dim3(1024), 0, s, scratch, nblocks);
  launch_pdl(k_fill_holes, dim3(nblocks), dim3(kHoleBlock), 0, s, p, dead_bits, scratch, nwords);
}

void aos_to_soa(const ParticleStateAoS* in, uint32_t n, ParticleArrays p, int nx, int ny, cudaStream_t s) {
  if (!n) return;
  k_aos_to_soa<<<grid_for(n), kBlock, 0, s>>>(in, n, p, nx, ny);
  GP_LAUNCH_CHECK();
}

void soa_to_aos(ParticleArrays p, uint32_t n, ParticleStateAoS* out, cudaStream_t s) {
  if (!n) return;
  k_soa_to_aos<<<grid_for(n), kBlock, 0, s>>>(p, n, out);
  GP_LAUNCH_CHECK();
}

}  // namespace kern
}  // namespace gample

