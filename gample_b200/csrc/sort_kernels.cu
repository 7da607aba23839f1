// sort_kernels.cu -- counting sort of the particles by cell (sm_100a).
//
// Key: the particle's cell in tile-major order (8 x 8-cell tiles, row-major
// over tiles, row-major inside a tile), so consecutive particles share a cell
// and a chunk of consecutive particles covers a compact box. Three passes:
// histogram (warp-aggregated atomics: lanes with equal keys add once),
// exclusive scan of the counts, scatter into the spare buffer (slots claimed
// with warp-aggregated atomics). The order inside a cell is unspecified.
//
// Particles in random order (just loaded or uploaded) take a staged scatter
// instead: each particle's six SoA words land in different 32-byte sectors
// when written one by one to random slots, so the staged path writes whole
// records into the spare buffer (its six arrays used as chunks of records)
// and then converts the records back to SoA with coalesced accesses. When
// the caller lends a second idle buffer (another species' spare), the
// records are padded to 32 bytes: each is then one whole, aligned sector,
// which the L2 writes back without first reading the rest of the sector from
// DRAM (a 24-byte record shares its sectors with records that arrive at
// other times). Otherwise they are 24-byte records.
//
// Nearly sorted particles (the periodic re-sort) take a block-local path:
// a block of kRsBlock consecutive particles, which covers a few cells plus
// the drift since the last sort, counts its particles per cell of a 32 x 32
// box around its middle particle in shared memory and adds each nonzero
// count to the global histogram once. Particles outside the box (strays:
// compaction fills holes with particles from the end of the store,
// re-injected particles) are counted with one global atomic each. In the
// scatter the block reserves each box cell's slots with one global atomic,
// orders its particles by box cell in shared memory and writes each cell's
// particles as one run of consecutive slots. Written straight from their
// source positions, a warp's 32 particles, spread over as many cells by the
// drift, would each land in a different 32-byte sector (27 sectors per
// store after 25 cycles at 64 particles per cell), and the L2 would read
// the rest of the partly written sectors back from DRAM (3x the traffic).
#include <cuda_runtime.h>

#include <climits>

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

__device__ __forceinline__ uint32_t xy_key(int ix, int iy, const KeyGeom& k) {
  const uint32_t tile = uint32_t((iy / kTile) * k.ntx + ix / kTile);
  return (tile * kTile + uint32_t(iy % kTile)) * kTile + uint32_t(ix % kTile);
}
__device__ __forceinline__ uint32_t cell_key(int32_t cell, const KeyGeom& k) {
  if (cell < 0) return k.nkeys;  // flagged particles (none after compaction) go last
  return xy_key(cell_ix(cell), cell_iy(cell), k);
}

// ---- block-local re-sort of nearly sorted particles
constexpr int kRsPer = 8;                    // particles per thread
constexpr int kRsBlock = kThreads * kRsPer;  // particles per block
constexpr int kRsBox = 32;                   // box of kRsBox x kRsBox cells
constexpr int kRsStray = -1, kRsNone = -2;   // bin of a particle outside the box / past the end

// Box origin of a block: its middle particle's cell, 15 cells to the left
// and below (a flagged middle particle leaves every particle a stray).
// Box origin of a block from its middle particle. Every thread reads the
// same cell (one broadcast load per warp, in flight with the thread's own
// loads), so no barrier waits on a global load to publish it.
__device__ __forceinline__ int2 rs_origin(const int32_t* cell, uint32_t n, uint32_t base) {
  const uint32_t rest = n - base;
  const int32_t c = __ldg(cell + base + (rest < uint32_t(kRsBlock) ? rest / 2 : uint32_t(kRsBlock / 2)));
  return c >= 0 ? make_int2(cell_ix(c) - (kRsBox / 2 - 1), cell_iy(c) - (kRsBox / 2 - 1))
                : make_int2(INT_MIN / 2, INT_MIN / 2);
}
__device__ __forceinline__ int rs_bin(int32_t c, int2 org) {
  if (c < 0) return kRsStray;
  const unsigned dx = unsigned(cell_ix(c) - org.x), dy = unsigned(cell_iy(c) - org.y);
  return dx < unsigned(kRsBox) && dy < unsigned(kRsBox) ? int(dy * kRsBox + dx) : kRsStray;
}
// Count the block's particles per box cell into bins (warp-aggregated
// shared atomics); strays are added to the global counts when counts != 0.
__device__ __forceinline__ void rs_count(const int32_t* __restrict__ cell, uint32_t n, uint32_t base, int2 org,
                                         const KeyGeom& g, uint32_t* bins, uint32_t* counts) {
  const int lane = threadIdx.x & 31;
  int32_t c[kRsPer];  // all loads first, so that they are in flight together
#pragma unroll
  for (int i = 0; i < kRsPer; ++i) {
    const uint32_t k = base + uint32_t(i * kThreads) + threadIdx.x;
    c[i] = k < n ? __ldg(cell + k) : INT_MIN;
  }
#pragma unroll
  for (int i = 0; i < kRsPer; ++i) {
    const int bin = c[i] != INT_MIN ? rs_bin(c[i], org) : kRsNone;
    const unsigned peers = __match_any_sync(0xffffffffu, bin);
    if (bin >= 0 && lane == __ffs(peers) - 1) atomicAdd(&bins[bin], uint32_t(__popc(peers)));
    if (counts && bin == kRsStray) atomicAdd(&counts[cell_key(c[i], g)], 1u);
  }
}

__global__ void __launch_bounds__(kThreads) k_rs_hist(const int32_t* cell, const SpeciesCounters* cnt, KeyGeom g,
                                                      uint32_t* counts) {
  __shared__ uint32_t bins[kRsBox * kRsBox];
  const uint32_t n = cnt->n, base = blockIdx.x * uint32_t(kRsBlock);
  if (base >= n) return;  // uniform over the block
  for (int b = threadIdx.x; b < kRsBox * kRsBox; b += kThreads) bins[b] = 0;
  const int2 org = rs_origin(cell, n, base);
  __syncthreads();
  rs_count(cell, n, base, org, g, bins, counts);
  __syncthreads();
  for (int b = threadIdx.x; b < kRsBox * kRsBox; b += kThreads)
    if (const uint32_t v = bins[b]) atomicAdd(&counts[xy_key(org.x + b % kRsBox, org.y + b / kRsBox, g)], v);
}

// Shared memory of k_rs_scatter: the staged particles (six words and the
// destination slot each, in box-cell order, strays last) and, per box cell
// and for the strays (entry kRsBins), the count / cursor, the first local
// position and the first global slot.
constexpr int kRsBins = kRsBox * kRsBox;
constexpr size_t kRsSmem = (size_t(kRsBlock) * 7 + 3 * size_t(kRsBins + 1)) * sizeof(uint32_t);

__global__ void __launch_bounds__(kThreads) k_rs_scatter(ParticleArrays src, ParticleArrays dst,
                                                         const SpeciesCounters* cnt, KeyGeom g, uint32_t* offsets) {
  extern __shared__ __align__(16) uint32_t rs_smem[];
  uint32_t* st = rs_smem;                   // [7][kRsBlock]: cell, ox, oy, vx, vy, vz, slot
  uint32_t* cur = st + 7 * kRsBlock;        // per bin: count, then cursor
  uint32_t* lbase = cur + (kRsBins + 1);    // per bin: first local position
  uint32_t* gbase = lbase + (kRsBins + 1);  // per box cell: first global slot
  __shared__ uint32_t s_warp[kThreads / 32];
  const uint32_t n = cnt->n, base = blockIdx.x * uint32_t(kRsBlock);
  if (base >= n) return;  // uniform over the block
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  for (int b = tid; b <= kRsBins; b += kThreads) cur[b] = 0;
  __syncthreads();
  const int2 org = rs_origin(src.cell, n, base);
  // this thread's particles, all loads first: cell, bin (strays: bin
  // kRsBins) and the five state words
  int32_t c[kRsPer];
  int bin[kRsPer];
  float w[5][kRsPer];
#pragma unroll
  for (int i = 0; i < kRsPer; ++i) {
    const uint32_t k = base + uint32_t(i * kThreads + tid);
    const bool in = k < n;
    c[i] = in ? __ldg(src.cell + k) : -1;
    w[0][i] = in ? __ldg(src.ox + k) : 0.0f;
    w[1][i] = in ? __ldg(src.oy + k) : 0.0f;
    w[2][i] = in ? __ldg(src.vx + k) : 0.0f;
    w[3][i] = in ? __ldg(src.vy + k) : 0.0f;
    w[4][i] = in ? __ldg(src.vz + k) : 0.0f;
  }
#pragma unroll
  for (int i = 0; i < kRsPer; ++i) {
    const uint32_t k = base + uint32_t(i * kThreads + tid);
    const int b = k < n ? rs_bin(c[i], org) : kRsNone;
    bin[i] = b == kRsStray ? kRsBins : b;
  }
#pragma unroll
  for (int i = 0; i < kRsPer; ++i) {
    const unsigned peers = __match_any_sync(0xffffffffu, bin[i]);
    if (bin[i] >= 0 && lane == __ffs(peers) - 1) atomicAdd(&cur[bin[i]], uint32_t(__popc(peers)));
  }
  __syncthreads();
  // exclusive scan of the counts into lbase (thread t: bins t*kEach ..),
  // the box cells' global slots reserved, cursors back to zero
  constexpr int kEach = (kRsBins + 1 + kThreads - 1) / kThreads;
  uint32_t v[kEach], run = 0;
#pragma unroll
  for (int e = 0; e < kEach; ++e) {
    const int b = tid * kEach + e;
    v[e] = b <= kRsBins ? cur[b] : 0u;
    run += v[e];
  }
  uint32_t incl = run;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) s_warp[wid] = incl;
  __syncthreads();
  uint32_t off = incl - run;
  for (int q = 0; q < wid; ++q) off += s_warp[q];
  const uint32_t total = [&] {
    uint32_t t = 0;
    for (int q = 0; q < kThreads / 32; ++q) t += s_warp[q];
    return t;
  }();
#pragma unroll
  for (int e = 0; e < kEach; ++e) {
    const int b = tid * kEach + e;
    if (b <= kRsBins) {
      lbase[b] = off;
      cur[b] = 0;
      if (b < kRsBins)
        gbase[b] = v[e] ? atomicAdd(&offsets[xy_key(org.x + b % kRsBox, org.y + b / kRsBox, g)], v[e]) : 0u;
    }
    off += v[e];
  }
  __syncthreads();
  // stage each particle at lbase[bin] + rank with its destination slot
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int i = 0; i < kRsPer; ++i) {
    const unsigned peers = __match_any_sync(0xffffffffu, bin[i]);
    const int leader = __ffs(peers) - 1;
    uint32_t r = 0;
    if (bin[i] >= 0 && lane == leader) r = atomicAdd(&cur[bin[i]], uint32_t(__popc(peers)));
    r = __shfl_sync(0xffffffffu, r, leader) + uint32_t(__popc(peers & lt));
    if (bin[i] >= 0) {
      const uint32_t lp = lbase[bin[i]] + r;
      const uint32_t slot = bin[i] < kRsBins ? gbase[bin[i]] + r : atomicAdd(&offsets[cell_key(c[i], g)], 1u);
      st[0 * kRsBlock + lp] = uint32_t(c[i]);
#pragma unroll
      for (int q = 0; q < 5; ++q) st[(q + 1) * kRsBlock + lp] = __float_as_uint(w[q][i]);
      st[6 * kRsBlock + lp] = slot;
    }
  }
  __syncthreads();
  // write out: consecutive local positions of one box cell go to
  // consecutive slots
  for (uint32_t j = tid; j < total; j += kThreads) {
    const uint32_t slot = st[6 * kRsBlock + j];
    dst.cell[slot] = int32_t(st[j]);
    dst.ox[slot] = __uint_as_float(st[1 * kRsBlock + j]);
    dst.oy[slot] = __uint_as_float(st[2 * kRsBlock + j]);
    dst.vx[slot] = __uint_as_float(st[3 * kRsBlock + j]);
    dst.vy[slot] = __uint_as_float(st[4 * kRsBlock + j]);
    dst.vz[slot] = __uint_as_float(st[5 * kRsBlock + j]);
  }
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

// One particle as a 24-byte record (8-byte aligned: three 64-bit stores).
struct __align__(8) Record {
  int32_t cell;
  float ox, oy, vx, vy, vz;
};
struct RecordChunks {  // slot s: chunk s / per, record s % per
  Record* c[6];
  uint32_t per;
};

__global__ void __launch_bounds__(kThreads) k_cs_scatter_rec(ParticleArrays src, RecordChunks dst,
                                                             const SpeciesCounters* cnt, KeyGeom g,
                                                             uint32_t* offsets) {
  const uint32_t n = cnt->n;
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  for (uint32_t base = (blockIdx.x * kThreads + threadIdx.x) & ~31u; base < n; base += gridDim.x * kThreads) {
    const uint32_t k = base + lane;
    const int32_t c = k < n ? src.cell[k] : 0;
    const uint32_t key = k < n ? cell_key(c, g) : kNoKey;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int leader = __ffs(peers) - 1;
    uint32_t slot = 0;
    if (key != kNoKey && lane == leader) slot = atomicAdd(&offsets[key], uint32_t(__popc(peers)));
    slot = __shfl_sync(0xffffffffu, slot, leader) + uint32_t(__popc(peers & lt));
    if (key != kNoKey) {
      Record r;
      r.cell = c;
      r.ox = src.ox[k];
      r.oy = src.oy[k];
      r.vx = src.vx[k];
      r.vy = src.vy[k];
      r.vz = src.vz[k];
      const uint32_t q = slot / dst.per;
      dst.c[q][slot - q * dst.per] = r;
    }
  }
}

// 32-byte records: slot s in chunk s / per, as two int4 (cell, ox, oy, vx),
// (vy, vz, 0, 0); the chunks start 32-byte aligned.
struct SectorChunks {
  int4* c[12];
  uint32_t per;
};

__global__ void __launch_bounds__(kThreads) k_cs_scatter_sec(ParticleArrays src, SectorChunks dst,
                                                             const SpeciesCounters* cnt, KeyGeom g,
                                                             uint32_t* offsets) {
  const uint32_t n = cnt->n;
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  for (uint32_t base = (blockIdx.x * kThreads + threadIdx.x) & ~31u; base < n; base += gridDim.x * kThreads) {
    const uint32_t k = base + lane;
    const int32_t c = k < n ? src.cell[k] : 0;
    const uint32_t key = k < n ? cell_key(c, g) : kNoKey;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int leader = __ffs(peers) - 1;
    uint32_t slot = 0;
    if (key != kNoKey && lane == leader) slot = atomicAdd(&offsets[key], uint32_t(__popc(peers)));
    slot = __shfl_sync(0xffffffffu, slot, leader) + uint32_t(__popc(peers & lt));
    if (key != kNoKey) {
      const int4 a = make_int4(c, __float_as_int(src.ox[k]), __float_as_int(src.oy[k]), __float_as_int(src.vx[k]));
      const int4 b = make_int4(__float_as_int(src.vy[k]), __float_as_int(src.vz[k]), 0, 0);
      const uint32_t q = slot / dst.per;
      int4* r = dst.c[q] + 2 * size_t(slot - q * dst.per);
      r[0] = a;
      r[1] = b;
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_sectors_to_soa(SectorChunks in, const SpeciesCounters* cnt,
                                                             ParticleArrays out) {
  const uint32_t n = cnt->n;
  for (uint32_t k = blockIdx.x * kThreads + threadIdx.x; k < n; k += gridDim.x * kThreads) {
    const uint32_t q = k / in.per;
    const int4* r = in.c[q] + 2 * size_t(k - q * in.per);
    const int4 a = r[0], b = r[1];
    out.cell[k] = a.x;
    out.ox[k] = __int_as_float(a.y);
    out.oy[k] = __int_as_float(a.z);
    out.vx[k] = __int_as_float(a.w);
    out.vy[k] = __int_as_float(b.x);
    out.vz[k] = __int_as_float(b.y);
  }
}

__global__ void __launch_bounds__(kThreads) k_records_to_soa(RecordChunks in, const SpeciesCounters* cnt,
                                                             ParticleArrays out) {
  const uint32_t n = cnt->n;
  for (uint32_t k = blockIdx.x * kThreads + threadIdx.x; k < n; k += gridDim.x * kThreads) {
    const uint32_t q = k / in.per;
    const Record r = in.c[q][k - q * in.per];
    out.cell[k] = r.cell;
    out.ox[k] = r.ox;
    out.oy[k] = r.oy;
    out.vx[k] = r.vx;
    out.vy[k] = r.vy;
    out.vz[k] = r.vz;
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

bool sort_by_cell_staged(GridDims g, ParticleArrays p, ParticleArrays spare, uint32_t capacity,
                         ParticleArrays extra, uint32_t extra_capacity, const SpeciesCounters* cnt,
                         uint32_t* scratch, uint32_t n_bound, cudaStream_t s) {
  // 32-byte records in the spare arrays and, if lent, the extra ones
  SectorChunks sc{};
  sc.per = uint32_t(size_t(capacity) * sizeof(int32_t) / 32);
  int nsc = 0;
  auto add_chunks = [&](const ParticleArrays& a) {
    void* arrs[6] = {a.cell, a.ox, a.oy, a.vx, a.vy, a.vz};
    for (void* q : arrs) {
      if (reinterpret_cast<uintptr_t>(q) % 32 != 0) return false;
      sc.c[nsc++] = static_cast<int4*>(q);
    }
    return true;
  };
  const bool sectors = n_bound > 0 && sc.per > 0 && extra_capacity >= capacity && add_chunks(spare) &&
                       add_chunks(extra) && size_t(n_bound) <= size_t(nsc) * sc.per;
  RecordChunks rc;
  rc.per = uint32_t(size_t(capacity) * sizeof(int32_t) / sizeof(Record));
  if (!sectors && (n_bound == 0 || rc.per == 0 || size_t(n_bound) > 6 * size_t(rc.per))) return false;
  rc.c[0] = reinterpret_cast<Record*>(spare.cell);
  rc.c[1] = reinterpret_cast<Record*>(spare.ox);
  rc.c[2] = reinterpret_cast<Record*>(spare.oy);
  rc.c[3] = reinterpret_cast<Record*>(spare.vx);
  rc.c[4] = reinterpret_cast<Record*>(spare.vy);
  rc.c[5] = reinterpret_cast<Record*>(spare.vz);
  const KeyGeom kg = geom(g);
  const uint32_t nk = kg.nkeys + 1;
  uint32_t* counts = scratch;
  uint32_t* offsets = scratch + nk;
  uint32_t* sums = scratch + 2 * size_t(nk);
  const uint32_t nb = (nk + kScanChunk - 1) / kScanChunk;
  GP_CUDA(cudaMemsetAsync(counts, 0, size_t(nk) * sizeof(uint32_t), s));
  k_cs_hist<<<grid_for(n_bound), kThreads, 0, s>>>(p.cell, cnt, kg, counts);
  GP_LAUNCH_CHECK();
  k_scan_local<<<nb, kScanThreads, 0, s>>>(counts, offsets, sums, nk);
  GP_LAUNCH_CHECK();
  k_scan_sums<<<1, kScanThreads, 0, s>>>(sums, nb);
  GP_LAUNCH_CHECK();
  k_scan_add<<<(nk + 255) / 256, 256, 0, s>>>(offsets, sums, nk);
  GP_LAUNCH_CHECK();
  if (sectors) {
    k_cs_scatter_sec<<<grid_for(n_bound), kThreads, 0, s>>>(p, sc, cnt, kg, offsets);
    GP_LAUNCH_CHECK();
    k_sectors_to_soa<<<grid_for(n_bound), kThreads, 0, s>>>(sc, cnt, p);
    GP_LAUNCH_CHECK();
  } else {
    k_cs_scatter_rec<<<grid_for(n_bound), kThreads, 0, s>>>(p, rc, cnt, kg, offsets);
    GP_LAUNCH_CHECK();
    k_records_to_soa<<<grid_for(n_bound), kThreads, 0, s>>>(rc, cnt, p);
    GP_LAUNCH_CHECK();
  }
  return true;
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
  const uint32_t nblocks = (n_bound + kRsBlock - 1) / kRsBlock;
  k_rs_hist<<<nblocks, kThreads, 0, s>>>(src.cell, cnt, kg, counts);
  GP_LAUNCH_CHECK();
  k_scan_local<<<nb, kScanThreads, 0, s>>>(counts, offsets, sums, nk);
  GP_LAUNCH_CHECK();
  k_scan_sums<<<1, kScanThreads, 0, s>>>(sums, nb);
  GP_LAUNCH_CHECK();
  k_scan_add<<<(nk + 255) / 256, 256, 0, s>>>(offsets, sums, nk);
  GP_LAUNCH_CHECK();
  static bool attr = [] {
    GP_CUDA(cudaFuncSetAttribute(k_rs_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kRsSmem)));
    return true;
  }();
  (void)attr;
  k_rs_scatter<<<nblocks, kThreads, kRsSmem, s>>>(src, dst, cnt, kg, offsets);
  GP_LAUNCH_CHECK();
}

}  // namespace kern
}  // namespace gample
