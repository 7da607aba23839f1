// particle_kernels.cu -- per-particle kernels of the PIC step (sm_100a).
//
//  k_push     gather (order 1/3/5 B-splines on the staggered grid) + Boris
//             rotation (order 2/4/6) + position update + boundary conditions
//             (src/Particle.mm:65-278), optionally fused with the charge /
//             current deposit of the new positions (src/Particle.mm:281-389)
//             so the next step needs no separate particle pass.
//  k_deposit  stand-alone deposit (src/Particle.mm:281-389).
//  compaction hole filling with the reference's permutation
//             (src/Particle.mm:893-966) driven by a dead bitmap.
#include <cuda_runtime.h>

#include <cstdio>

#include "device.hpp"
#include "kernels.hpp"
#include "pic_common.cuh"

namespace gample {
namespace kern {

namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ uint32_t warp_sum(uint32_t v) { return __reduce_add_sync(0xffffffffu, v); }
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// In-range test used by the bounds-checked stencil paths.
__device__ __forceinline__ bool in_box(int i, int j, int w, int h) { return i >= 0 && j >= 0 && i < w && j < h; }

// Deposit the weights of one particle (already evaluated) into the targets.
// CHECKED skips stencil nodes outside the arrays: a particle exactly on the
// far boundary (x = Xmax from a loader draw of 1.0) touches one node past the
// array with weight zero in the reference (src/Particle.mm:357-373).
template <int ORDER, bool DET, bool CUR, bool CHECKED = false>
__device__ __forceinline__ void deposit_weights(const GridDims& g, const Stagger& sx, const Stagger& sy,
                                                const float (&wxn)[ORDER + 1], const float (&wxh)[ORDER + 1],
                                                const float (&wyn)[ORDER + 1], const float (&wyh)[ORDER + 1],
                                                float scale, float vx, float vy, const DepositTargets& d) {
  const int ngb = g.ngb, nx = g.nx;
  // rho: node x (i2) x node y (j1): src/Particle.mm:360-362
  const int rbase = (sy.node - ngb) * (nx + 1) + (sx.node - ngb);
#pragma unroll
  for (int i = 0; i <= ORDER; ++i)
#pragma unroll
    for (int j = 0; j <= ORDER; ++j) {
      if (CHECKED && !in_box(sx.node - ngb + i, sy.node - ngb + j, nx + 1, g.ny + 1)) continue;
      const float w = __fmul_rn(wxn[i], wyn[j]);
      if constexpr (DET)
        red_add(d.acc_rho + rbase + i + j * (nx + 1), quant40(w));
      else
        red_add(d.rho + rbase + i + j * (nx + 1), __fmul_rn(w, scale));
    }
  if constexpr (CUR) {
    // jx: half x (i1) x node y (j1); jy: node x (i2) x half y (j2):
    // src/Particle.mm:365-372
    const int xbase = (sy.node - ngb) * (nx + 2) + (sx.half - ngb + 1);
    const int ybase = (sy.half - ngb + 1) * (nx + 1) + (sx.node - ngb);
    constexpr float inv_c = float(1.0 / 2.99792458e10);
    const float ux = __fmul_rn(vx, inv_c), uy = __fmul_rn(vy, inv_c);
#pragma unroll
    for (int i = 0; i <= ORDER; ++i)
#pragma unroll
      for (int j = 0; j <= ORDER; ++j) {
        const float wx = __fmul_rn(wxh[i], wyn[j]);
        const float wy = __fmul_rn(wxn[i], wyh[j]);
        const bool okx = !CHECKED || in_box(sx.half - ngb + 1 + i, sy.node - ngb + j, nx + 2, g.ny + 1);
        const bool oky = !CHECKED || in_box(sx.node - ngb + i, sy.half - ngb + 1 + j, nx + 1, g.ny + 2);
        if constexpr (DET) {
          if (okx) red_add(d.acc_jx + xbase + i + j * (nx + 2), quant40(__fmul_rn(wx, ux)));
          if (oky) red_add(d.acc_jy + ybase + i + j * (nx + 1), quant40(__fmul_rn(wy, uy)));
        } else {
          if (okx) red_add(d.jx + xbase + i + j * (nx + 2), __fmul_rn(__fmul_rn(wx, scale), vx));
          if (oky) red_add(d.jy + ybase + i + j * (nx + 1), __fmul_rn(__fmul_rn(wy, scale), vy));
        }
      }
  }
}

// Reflection of a coordinate (cell, offset) about the integer plane B:
// x' = 2B - x (src/Particle.mm:246-269).
__device__ __forceinline__ void reflect(int& i, float& o, int B) {
  if (o > 0.0f) {
    i = 2 * B - i - 1;
    o = __fsub_rn(1.0f, o);
    if (o >= 1.0f) {
      o = 0.0f;
      i += 1;
    }
  } else {
    i = 2 * B - i;
  }
}

// Move by d cells (float), keeping (i, o) normalised with o in [0, 1).
// Returns false for a non-finite or absurd displacement.
__device__ __forceinline__ bool advance(int& i, float& o, float v, float cst) {
  const float f = o + v * cst;
  if (!(fabsf(f) < 1.0e7f)) return false;
  const float fl = floorf(f);
  float r = __fsub_rn(f, fl);
  int di = __float2int_rn(fl);
  if (r >= 1.0f) {  // f slightly below an integer rounds to 1 - ulp -> 1
    r = 0.0f;
    di += 1;
  }
  i += di;
  o = r;
  return true;
}

// Gather with every tap bounds-checked (particles not strictly inside the
// grid, e.g. exactly on the far boundary after loading).
template <int ORDER, bool BZU>
__device__ __noinline__ void gather_checked(const GridDims& g, const FieldPtrs& f, const Stagger& sx,
                                            const Stagger& sy, const float (&wxn)[ORDER + 1],
                                            const float (&wxh)[ORDER + 1], const float (&wyn)[ORDER + 1],
                                            const float (&wyh)[ORDER + 1], float& Epx, float& Epy, float& Bpz) {
  const int ngb = g.ngb, nx = g.nx, ny = g.ny;
  for (int i = 0; i <= ORDER; ++i)
    for (int j = 0; j <= ORDER; ++j) {
      int ii = sx.half - ngb + 1 + i, jj = sy.node - ngb + j;
      if (in_box(ii, jj, nx + 2, ny + 1)) Epx += (wxh[i] * wyn[j]) * f.Ex[ii + jj * (nx + 2)];
      ii = sx.node - ngb + i;
      jj = sy.half - ngb + 1 + j;
      if (in_box(ii, jj, nx + 1, ny + 2)) Epy += (wxn[i] * wyh[j]) * f.Ey[ii + jj * (nx + 1)];
      if (!BZU) {
        ii = sx.half - ngb + 1 + i;
        jj = sy.half - ngb + 1 + j;
        if (in_box(ii, jj, nx + 2, ny + 2)) Bpz += (wxh[i] * wyh[j]) * f.Bz[ii + jj * (nx + 2)];
      }
    }
}

template <int ORDER, bool DEP, bool DET, bool CUR, bool BZU>
__global__ void __launch_bounds__(kBlock) k_push(GridDims g, ParticleArrays p, FieldPtrs f, PushConsts c,
                                                 int boris_order, DepositTargets d, SpeciesCounters* cnt,
                                                 uint32_t* dead_bits) {
  const uint32_t n = cnt->n;
  const int lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  uint32_t wcount[4] = {0, 0, 0, 0}, ninvalid = 0, ndead = 0;
  double ke = 0.0;
  const int ngb = g.ngb, nx = g.nx;
  for (uint32_t base = warp * 32u; base < n; base += nwarps * 32u) {
    const uint32_t k = base + lane;
    int fl = 0;
    if (k < n) {
      const int32_t cell = p.cell[k];
      if (cell < 0) {
        fl = -cell;  // already flagged (not yet compacted): keep the flag
      } else {
        int ix = cell_ix(cell), iy = cell_iy(cell);
        float ox = p.ox[k], oy = p.oy[k];
        float vx = p.vx[k], vy = p.vy[k], vz = p.vz[k];
        const Stagger sx = stagger(ix, ox), sy = stagger(iy, oy);
        float wxn[ORDER + 1], wxh[ORDER + 1], wyn[ORDER + 1], wyh[ORDER + 1];
        shape<ORDER>(sx.hnode, wxn);
        shape<ORDER>(sx.hhalf, wxh);
        shape<ORDER>(sy.hnode, wyn);
        shape<ORDER>(sy.hhalf, wyh);
        // Gather (src/Particle.mm:142-154): Ex half-x/node-y, Ey node-x/half-y,
        // Bz half-x/half-y.
        float Epx = 0.0f, Epy = 0.0f, Bpz = 0.0f;
        const bool interior = ix >= ngb && ix < ngb + g.ngx && iy >= ngb && iy < ngb + g.ngy;
        if (interior) {
          const float* exr = f.Ex + (sy.node - ngb) * (nx + 2) + (sx.half - ngb + 1);
          const float* eyr = f.Ey + (sy.half - ngb + 1) * (nx + 1) + (sx.node - ngb);
          const float* bzr = f.Bz + (sy.half - ngb + 1) * (nx + 2) + (sx.half - ngb + 1);
#pragma unroll
          for (int i = 0; i <= ORDER; ++i)
#pragma unroll
            for (int j = 0; j <= ORDER; ++j) {
              Epx += (wxh[i] * wyn[j]) * __ldg(exr + i + j * (nx + 2));
              Epy += (wxn[i] * wyh[j]) * __ldg(eyr + i + j * (nx + 1));
              if constexpr (!BZU) Bpz += (wxh[i] * wyh[j]) * __ldg(bzr + i + j * (nx + 2));
            }
        } else {
          gather_checked<ORDER, BZU>(g, f, sx, sy, wxn, wxh, wyn, wyh, Epx, Epy, Bpz);
        }
        if constexpr (BZU) Bpz = c.bz_uniform;
        // Boris push (src/Particle.mm:157-209); Ez, Bx, By are identically
        // zero in the reference's gather (:134-139).
        float etx = c.constE * Epx, ety = c.constE * Epy;
        float btz = c.constB * Bpz;
        const float btbt = btz * btz;
        if (boris_order == 4) {
          const float fN1 = 1.0f + btbt / 3.0f;
          etx *= fN1;
          ety *= fN1;
          btz *= fN1;
        } else if (boris_order == 6) {
          const float fN1 = 1.0f + btbt / 3.0f + 2.0f * btbt * btbt / 15.0f;
          etx *= fN1;
          ety *= fN1;
          btz *= fN1;
        }
        const float umx = vx + etx, umy = vy + ety, umz = vz;
        const float v0x = umx + umy * btz;
        const float v0y = umy - umx * btz;
        const float ssz = 2.0f * btz / (1.0f + btbt);
        const float upx = umx + v0y * ssz;
        const float upy = umy - v0x * ssz;
        vx = upx + c.constE * Epx;
        vy = upy + c.constE * Epy;
        vz = umz;
        // Position update and boundary conditions (src/Particle.mm:212-269).
        const bool okx = advance(ix, ox, vx, c.constX);
        const bool oky = advance(iy, oy, vy, c.constY);
        if (!(okx && oky) || !isfinite(vz)) {
          fl = 5;
        } else {
          if (c.bc[0] == 0) ix = ngb + (((ix - ngb) % g.ngx) + g.ngx) % g.ngx;
          if (c.bc[2] == 0) iy = ngb + (((iy - ngb) % g.ngy) + g.ngy) % g.ngy;
          if (c.bc[0] == 1 && ix < ngb) fl = 1;
          if (c.bc[1] == 1 && ix >= ngb + g.ngx) fl = 2;
          if (c.bc[2] == 1 && iy < ngb) fl = 3;
          if (c.bc[3] == 1 && iy >= ngb + g.ngy) fl = 4;
          if (c.bc[0] == 2 && ix < ngb) {
            reflect(ix, ox, ngb);
            vx = -vx;
          }
          if (c.bc[1] == 2 && ix >= ngb + g.ngx) {
            reflect(ix, ox, ngb + g.ngx);
            vx = -vx;
          }
          if (c.bc[2] == 2 && iy < ngb) {
            reflect(iy, oy, ngb);
            vy = -vy;
          }
          if (c.bc[3] == 2 && iy >= ngb + g.ngy) {
            reflect(iy, oy, ngb + g.ngy);
            vy = -vy;
          }
          // A live particle must stay on the grid, or its next stencil would
          // leave the arrays (possible only for displacements of more than
          // the domain in one step).
          if (fl == 0 && (ix < ngb || ix >= ngb + g.ngx || iy < ngb || iy >= ngb + g.ngy)) fl = 5;
        }
        p.vx[k] = vx;
        p.vy[k] = vy;
        p.vz[k] = vz;
        if (fl == 0) {
          p.cell[k] = pack_cell(ix, iy);
          p.ox[k] = ox;
          p.oy[k] = oy;
          // kinetic energy, src/Particle.mm:980-982
          const float vv = __fadd_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)), __fmul_rn(vz, vz));
          ke += (c.ke_half_m * double(vv)) * c.ke_w;
          if constexpr (DEP) {
            const Stagger nsx = stagger(ix, ox), nsy = stagger(iy, oy);
            shape<ORDER>(nsx.hnode, wxn);
            shape<ORDER>(nsy.hnode, wyn);
            if constexpr (CUR) {
              shape<ORDER>(nsx.hhalf, wxh);
              shape<ORDER>(nsy.hhalf, wyh);
            }
            deposit_weights<ORDER, DET, CUR>(g, nsx, nsy, wxn, wxh, wyn, wyh, c.scale, vx, vy, d);
          }
        } else {
          p.cell[k] = -fl;
        }
      }
      if (fl) {  // includes particles flagged before this push and not yet compacted
        ndead++;
        if (fl <= 4)
          wcount[fl - 1]++;
        else
          ninvalid++;
      }
    }
    const uint32_t bits = __ballot_sync(0xffffffffu, fl != 0);
    if (lane == 0) dead_bits[base >> 5] = bits;
  }
  // Warp-aggregated counters.
  const uint32_t s_dead = warp_sum(ndead);
  const uint32_t s_w0 = warp_sum(wcount[0]), s_w1 = warp_sum(wcount[1]);
  const uint32_t s_w2 = warp_sum(wcount[2]), s_w3 = warp_sum(wcount[3]);
  const uint32_t s_inv = warp_sum(ninvalid);
  const double s_ke = warp_sum(ke);
  if (lane == 0) {
    if (s_dead) atomicAdd(&cnt->n_dead, s_dead);
    if (s_w0) atomicAdd(&cnt->wall[0], s_w0);
    if (s_w1) atomicAdd(&cnt->wall[1], s_w1);
    if (s_w2) atomicAdd(&cnt->wall[2], s_w2);
    if (s_w3) atomicAdd(&cnt->wall[3], s_w3);
    if (s_inv) atomicAdd(&cnt->invalid, s_inv);
    if (s_ke != 0.0) atomicAdd(&cnt->ke, s_ke);
  }
}

template <int ORDER, bool DET, bool CUR>
__global__ void __launch_bounds__(kBlock) k_deposit(GridDims g, ParticleArrays p, float scale, DepositTargets d,
                                                    const SpeciesCounters* cnt, bool injected_only) {
  const uint32_t n = cnt->n;
  const uint32_t first = injected_only ? n - cnt->n_injected : 0u;
  for (uint32_t k = first + blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int32_t cell = p.cell[k];
    if (cell < 0) continue;
    const Stagger sx = stagger(cell_ix(cell), p.ox[k]), sy = stagger(cell_iy(cell), p.oy[k]);
    float wxn[ORDER + 1], wxh[ORDER + 1], wyn[ORDER + 1], wyh[ORDER + 1];
    shape<ORDER>(sx.hnode, wxn);
    shape<ORDER>(sy.hnode, wyn);
    float vx = 0.0f, vy = 0.0f;
    if constexpr (CUR) {
      shape<ORDER>(sx.hhalf, wxh);
      shape<ORDER>(sy.hhalf, wyh);
      vx = p.vx[k];
      vy = p.vy[k];
    }
    const int ix = cell_ix(cell), iy = cell_iy(cell);
    if (ix >= g.ngb && ix < g.ngb + g.ngx && iy >= g.ngb && iy < g.ngb + g.ngy)
      deposit_weights<ORDER, DET, CUR>(g, sx, sy, wxn, wxh, wyn, wyh, scale, vx, vy, d);
    else
      deposit_weights<ORDER, DET, CUR, true>(g, sx, sy, wxn, wxh, wyn, wyh, scale, vx, vy, d);
  }
}

template <int ORDER, bool DEP, bool DET, bool CUR>
void launch_push_bz(bool bzu, dim3 grid, cudaStream_t s, GridDims g, ParticleArrays p, FieldPtrs f, PushConsts c,
                    int boris, DepositTargets d, SpeciesCounters* cnt, uint32_t* bits) {
  if (bzu)
    k_push<ORDER, DEP, DET, CUR, true><<<grid, kBlock, 0, s>>>(g, p, f, c, boris, d, cnt, bits);
  else
    k_push<ORDER, DEP, DET, CUR, false><<<grid, kBlock, 0, s>>>(g, p, f, c, boris, d, cnt, bits);
}

template <int ORDER>
void launch_push_order(bool dep, bool det, bool cur, bool bzu, dim3 grid, cudaStream_t s, GridDims g,
                       ParticleArrays p, FieldPtrs f, PushConsts c, int boris, DepositTargets d,
                       SpeciesCounters* cnt, uint32_t* bits) {
  if (!dep)
    launch_push_bz<ORDER, false, false, false>(bzu, grid, s, g, p, f, c, boris, d, cnt, bits);
  else if (det)
    cur ? launch_push_bz<ORDER, true, true, true>(bzu, grid, s, g, p, f, c, boris, d, cnt, bits)
        : launch_push_bz<ORDER, true, true, false>(bzu, grid, s, g, p, f, c, boris, d, cnt, bits);
  else
    cur ? launch_push_bz<ORDER, true, false, true>(bzu, grid, s, g, p, f, c, boris, d, cnt, bits)
        : launch_push_bz<ORDER, true, false, false>(bzu, grid, s, g, p, f, c, boris, d, cnt, bits);
}

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

__device__ __forceinline__ uint32_t hole_mask(const uint32_t* bits, uint32_t w, uint32_t nl) {
  return bits[w] & live_mask_range(w, 0, nl);
}

__global__ void __launch_bounds__(kHoleBlock) k_hole_count(const uint32_t* bits, uint32_t* scratch) {
  __shared__ uint32_t s_red[kHoleBlock / 32];
  const uint32_t nl = scratch[0];
  const uint32_t nw = (nl + 31u) >> 5;
  const uint32_t w0 = blockIdx.x * kWordsPerBlock + threadIdx.x * kWordsPerThread;
  uint32_t c = 0;
#pragma unroll
  for (int t = 0; t < kWordsPerThread; ++t)
    if (w0 + t < nw) c += __popc(hole_mask(bits, w0 + t, nl));
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

__global__ void __launch_bounds__(kHoleBlock) k_fill_holes(ParticleArrays p, const uint32_t* bits,
                                                           const uint32_t* scratch) {
  __shared__ uint32_t s_warp[kHoleBlock / 32];
  const uint32_t nl = scratch[0];
  const uint32_t nw = (nl + 31u) >> 5;
  const uint32_t w0 = blockIdx.x * kWordsPerBlock + threadIdx.x * kWordsPerThread;
  uint32_t m[kWordsPerThread];
  uint32_t c = 0;
#pragma unroll
  for (int t = 0; t < kWordsPerThread; ++t) {
    m[t] = (w0 + t < nw) ? hole_mask(bits, w0 + t, nl) : 0u;
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
  uint32_t rank = scratch[16 + blockIdx.x] + s_warp[wid] + incl - c;
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

__global__ void k_aos_to_soa(const ParticleStateAoS* in, uint32_t n, ParticleArrays p) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const ParticleStateAoS r = in[k];
    const float fx = floorf(r.x), fy = floorf(r.y);
    int ix = int(fx), iy = int(fy);
    bool ok = isfinite(r.x) && isfinite(r.y) && ix >= 0 && iy >= 0 && ix < 65536 && iy < 32768;
    if (r.piflag > 0 || !ok) {
      p.cell[k] = -(r.piflag > 0 ? (r.piflag <= 5 ? r.piflag : 5) : 5);
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

void push(int order, int boris_order, bool dep, bool det, bool cur, bool bzu, GridDims g, ParticleArrays p,
          FieldPtrs f, PushConsts c, DepositTargets d, SpeciesCounters* cnt, uint32_t* dead_bits,
          uint32_t n_bound, cudaStream_t s) {
  // Zero the per-push counters (everything after n).
  GP_CUDA(cudaMemsetAsync(&cnt->n_dead, 0, sizeof(SpeciesCounters) - offsetof(SpeciesCounters, n_dead), s));
  if (n_bound == 0) return;
  dim3 grid(grid_for(n_bound));
  switch (order) {
    case 1: launch_push_order<1>(dep, det, cur, bzu, grid, s, g, p, f, c, boris_order, d, cnt, dead_bits); break;
    case 3: launch_push_order<3>(dep, det, cur, bzu, grid, s, g, p, f, c, boris_order, d, cnt, dead_bits); break;
    case 5: launch_push_order<5>(dep, det, cur, bzu, grid, s, g, p, f, c, boris_order, d, cnt, dead_bits); break;
    default: throw std::invalid_argument("WeightingOrder must be 1, 3 or 5");
  }
  GP_LAUNCH_CHECK();
}

void deposit(int order, bool det, bool cur, GridDims g, ParticleArrays p, float scale, DepositTargets d,
             const SpeciesCounters* cnt, uint32_t n_bound, bool injected_only, cudaStream_t s) {
  if (n_bound == 0) return;
  dim3 grid(grid_for(n_bound));
#define GP_DEP(O)                                                                             \
  if (det)                                                                                    \
    cur ? k_deposit<O, true, true><<<grid, kBlock, 0, s>>>(g, p, scale, d, cnt, injected_only)               \
        : k_deposit<O, true, false><<<grid, kBlock, 0, s>>>(g, p, scale, d, cnt, injected_only);             \
  else                                                                                        \
    cur ? k_deposit<O, false, true><<<grid, kBlock, 0, s>>>(g, p, scale, d, cnt, injected_only)              \
        : k_deposit<O, false, false><<<grid, kBlock, 0, s>>>(g, p, scale, d, cnt, injected_only);
  switch (order) {
    case 1: GP_DEP(1) break;
    case 3: GP_DEP(3) break;
    case 5: GP_DEP(5) break;
    default: throw std::invalid_argument("WeightingOrder must be 1, 3 or 5");
  }
#undef GP_DEP
  GP_LAUNCH_CHECK();
}

size_t compact_scratch_words(uint32_t n_bound) { return 16 + size_t(kMaxScanBlocks) + size_t(n_bound) + 32; }

void compact(ParticleArrays p, SpeciesCounters* cnt, const uint32_t* dead_bits, uint32_t* scratch,
             uint32_t n_bound, cudaStream_t s) {
  if (n_bound == 0) return;
  k_compact_tail<<<1, 1024, 0, s>>>(cnt, dead_bits, scratch);
  GP_LAUNCH_CHECK();
  const uint32_t nwords = (n_bound + 31u) / 32u;
  const uint32_t nblocks = (nwords + kWordsPerBlock - 1) / kWordsPerBlock;
  k_hole_count<<<nblocks, kHoleBlock, 0, s>>>(dead_bits, scratch);
  GP_LAUNCH_CHECK();
  k_scan_blocks<<<1, 1024, 0, s>>>(scratch, nblocks);
  GP_LAUNCH_CHECK();
  k_fill_holes<<<nblocks, kHoleBlock, 0, s>>>(p, dead_bits, scratch);
  GP_LAUNCH_CHECK();
}

void aos_to_soa(const ParticleStateAoS* in, uint32_t n, ParticleArrays p, cudaStream_t s) {
  if (!n) return;
  k_aos_to_soa<<<grid_for(n), kBlock, 0, s>>>(in, n, p);
  GP_LAUNCH_CHECK();
}

void soa_to_aos(ParticleArrays p, uint32_t n, ParticleStateAoS* out, cudaStream_t s) {
  if (!n) return;
  k_soa_to_aos<<<grid_for(n), kBlock, 0, s>>>(p, n, out);
  GP_LAUNCH_CHECK();
}

}  // namespace kern
}  // namespace gample
