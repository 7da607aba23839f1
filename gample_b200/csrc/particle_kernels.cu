// particle_kernels.cu -- per-particle kernels of the PIC step (sm_100a).
//
//  k_pic<PUSH=true>   gather (order 1/3/5 B-splines on the staggered grid) +
//                     Boris rotation (order 2/4/6) + position update +
//                     boundary conditions (src/Particle.mm:65-278), optionally
//                     fused with the charge/current deposit of the new
//                     positions (src/Particle.mm:281-389).
//  k_pic<PUSH=false>  deposit of the current positions (src/Particle.mm:281-389).
//  k_sort_*           counting sort of the particles by spatial tile.
//
// Work decomposition: one CTA per chunk of kChunk consecutive particles.
// Because the particles are tile-sorted, a chunk covers a small box of cells;
// the CTA stages the field window of that box (Ex, Ey, Bz) in shared memory
// and accumulates its deposit in a shared-memory window that is flushed with
// one global atomic per touched node (FP64 per species, or exact int64 in the
// deterministic mode). Chunks whose box does not fit (unsorted or drifted
// particles) fall back to direct global gathers/atomics, per chunk; particles
// not strictly inside the grid use bounds-checked stencils.
#include <cuda_runtime.h>

#include <climits>
#include <cstdio>

#include "device.hpp"
#include "kernels.hpp"
#include "pic_common.cuh"

namespace gample {
namespace kern {

namespace {

constexpr int kThreads = 256;
constexpr int kPer = 8;                      // particles per thread
constexpr int kChunk = kThreads * kPer;      // particles per CTA
constexpr int kWin = 1600;                   // entries of a shared-memory window (e.g. 40 x 40)
constexpr int kMargin = 2;                   // deposit-window margin for the motion of one step (cells)

__device__ __forceinline__ uint32_t warp_sum(uint32_t v) { return __reduce_add_sync(0xffffffffu, v); }
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ bool in_box(int i, int j, int w, int h) { return i >= 0 && j >= 0 && i < w && j < h; }

template <bool DET>
struct AccT {
  using type = float;
};
template <>
struct AccT<true> {
  using type = long long;
};

__device__ __forceinline__ void gadd(double* p, float v) { atomicAdd(p, double(v)); }
__device__ __forceinline__ void gadd(long long* p, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(v));
}
__device__ __forceinline__ void sadd(float* p, float v) { atomicAdd(p, v); }
__device__ __forceinline__ void sadd(long long* p, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(v));
}

// Contribution of one stencil node (rho and the two currents).
template <bool DET>
struct Contrib {
  using T = typename AccT<DET>::type;
  __device__ __forceinline__ static T rho(float w, float scale) {
    if constexpr (DET)
      return quant40(w);
    else
      return __fmul_rn(w, scale);
  }
  // current: fast mode (w * scale) * v (src/Particle.mm:368, 371); deterministic
  // mode quantises w * v / c.
  __device__ __forceinline__ static T cur(float w, float scale, float v, float u) {
    if constexpr (DET)
      return quant40(__fmul_rn(w, u));
    else
      return __fmul_rn(__fmul_rn(w, scale), v);
  }
};

struct Window {  // shared-memory windows of one CTA (array-index coordinates)
  int use;       // 1: staged windows valid for this chunk
  int mnx, mny, mxx, mxy;
  int gx0, gy0, gw, gh;  // gather window (origin, size)
  int dx0, dy0, dw, dh;  // deposit window
};

// Deposit one particle's weights. WIN: into the shared-memory window;
// otherwise global (CHECKED skips nodes outside the arrays, which carry
// weight zero for a particle exactly on the far wall, src/Particle.mm:357-373).
template <int ORDER, bool DET, bool CUR, bool WIN, bool CHECKED>
__device__ __forceinline__ void deposit_one(const GridDims& g, const Window& w, const Stagger& sx, const Stagger& sy,
                                            const float (&wxn)[ORDER + 1], const float (&wxh)[ORDER + 1],
                                            const float (&wyn)[ORDER + 1], const float (&wyh)[ORDER + 1],
                                            float scale, float vx, float vy, const DepositTargets& d,
                                            typename AccT<DET>::type* sRho, typename AccT<DET>::type* sJx,
                                            typename AccT<DET>::type* sJy) {
  using C = Contrib<DET>;
  const int ngb = g.ngb, nx = g.nx, ny = g.ny;
  const int rc = sx.node - ngb, rr = sy.node - ngb;  // rho / jy column base, rho / jx row base
#pragma unroll
  for (int i = 0; i <= ORDER; ++i)
#pragma unroll
    for (int j = 0; j <= ORDER; ++j) {
      const auto v = C::rho(__fmul_rn(wxn[i], wyn[j]), scale);
      if constexpr (WIN) {
        sadd(sRho + (rc + i - w.dx0) + (rr + j - w.dy0) * w.dw, v);
      } else {
        if (CHECKED && !in_box(rc + i, rr + j, nx + 1, ny + 1)) continue;
        if constexpr (DET)
          gadd(d.acc_rho + (rc + i) + (rr + j) * (nx + 1), v);
        else
          gadd(d.f64_rho + (rc + i) + (rr + j) * (nx + 1), v);
      }
    }
  if constexpr (CUR) {
    constexpr float inv_c = float(1.0 / 2.99792458e10);
    const float ux = __fmul_rn(vx, inv_c), uy = __fmul_rn(vy, inv_c);
    const int xc = sx.half - ngb + 1, yr = sy.half - ngb + 1;  // jx column base, jy row base
#pragma unroll
    for (int i = 0; i <= ORDER; ++i)
#pragma unroll
      for (int j = 0; j <= ORDER; ++j) {
        const auto a = C::cur(__fmul_rn(wxh[i], wyn[j]), scale, vx, ux);
        const auto b = C::cur(__fmul_rn(wxn[i], wyh[j]), scale, vy, uy);
        if constexpr (WIN) {
          sadd(sJx + (xc + i - w.dx0) + (rr + j - w.dy0) * w.dw, a);
          sadd(sJy + (rc + i - w.dx0) + (yr + j - w.dy0) * w.dw, b);
        } else {
          const bool oka = !CHECKED || in_box(xc + i, rr + j, nx + 2, ny + 1);
          const bool okb = !CHECKED || in_box(rc + i, yr + j, nx + 1, ny + 2);
          if constexpr (DET) {
            if (oka) gadd(d.acc_jx + (xc + i) + (rr + j) * (nx + 2), a);
            if (okb) gadd(d.acc_jy + (rc + i) + (yr + j) * (nx + 1), b);
          } else {
            if (oka) gadd(d.f64_jx + (xc + i) + (rr + j) * (nx + 2), a);
            if (okb) gadd(d.f64_jy + (rc + i) + (yr + j) * (nx + 1), b);
          }
        }
      }
  }
}

// Gather Ex, Ey (and Bz) for one particle (src/Particle.mm:142-154).
// WIN: from the staged windows; CHECKED: global with bounds checks.
template <int ORDER, bool BZU, bool WIN, bool CHECKED>
__device__ __forceinline__ void gather(const GridDims& g, const FieldPtrs& f, const Window& w, const Stagger& sx,
                                       const Stagger& sy, const float (&wxn)[ORDER + 1],
                                       const float (&wxh)[ORDER + 1], const float (&wyn)[ORDER + 1],
                                       const float (&wyh)[ORDER + 1], const float* sEx, const float* sEy,
                                       const float* sBz, float& Epx, float& Epy, float& Bpz) {
  const int ngb = g.ngb, nx = g.nx, ny = g.ny;
  const int hc = sx.half - ngb + 1, nc = sx.node - ngb;   // Ex/Bz and Ey column bases
  const int nr = sy.node - ngb, hr = sy.half - ngb + 1;   // Ex and Ey/Bz row bases
#pragma unroll
  for (int i = 0; i <= ORDER; ++i)
#pragma unroll
    for (int j = 0; j <= ORDER; ++j) {
      if constexpr (WIN) {
        Epx += (wxh[i] * wyn[j]) * sEx[(hc + i - w.gx0) + (nr + j - w.gy0) * w.gw];
        Epy += (wxn[i] * wyh[j]) * sEy[(nc + i - w.gx0) + (hr + j - w.gy0) * w.gw];
        if constexpr (!BZU) Bpz += (wxh[i] * wyh[j]) * sBz[(hc + i - w.gx0) + (hr + j - w.gy0) * w.gw];
      } else {
        if (!CHECKED || in_box(hc + i, nr + j, nx + 2, ny + 1))
          Epx += (wxh[i] * wyn[j]) * __ldg(f.Ex + (hc + i) + (nr + j) * (nx + 2));
        if (!CHECKED || in_box(nc + i, hr + j, nx + 1, ny + 2))
          Epy += (wxn[i] * wyh[j]) * __ldg(f.Ey + (nc + i) + (hr + j) * (nx + 1));
        if constexpr (!BZU)
          if (!CHECKED || in_box(hc + i, hr + j, nx + 2, ny + 2))
            Bpz += (wxh[i] * wyh[j]) * __ldg(f.Bz + (hc + i) + (hr + j) * (nx + 2));
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

// Move by v*cst cells keeping (i, o) normalised with o in [0, 1).
// Returns false for a non-finite or absurd displacement.
__device__ __forceinline__ bool advance(int& i, float& o, float v, float cst) {
  const float fpos = o + v * cst;
  if (!(fabsf(fpos) < 1.0e7f)) return false;
  const float fl = floorf(fpos);
  float r = __fsub_rn(fpos, fl);
  int di = __float2int_rn(fl);
  if (r >= 1.0f) {  // fpos slightly below an integer rounds to 1 - ulp -> 1
    r = 0.0f;
    di += 1;
  }
  i += di;
  o = r;
  return true;
}

__device__ __forceinline__ bool interior(const GridDims& g, int ix, int iy) {
  return ix >= g.ngb && ix < g.ngb + g.ngx && iy >= g.ngb && iy < g.ngb + g.ngy;
}

template <int ORDER, bool PUSH, bool DEP, bool DET, bool BZU>
__host__ __device__ constexpr size_t smem_bytes(bool cur) {
  return (PUSH ? (BZU ? 2 : 3) * size_t(kWin) * sizeof(float) : 0) +
         (DEP ? (cur ? 3 : 1) * size_t(kWin) * (DET ? sizeof(long long) : sizeof(float)) : 0);
}

template <int ORDER, bool PUSH, bool DEP, bool DET, bool CUR, bool BZU>
__global__ void __launch_bounds__(kThreads) k_pic(GridDims g, ParticleArrays p, FieldPtrs f, PushConsts c,
                                                  int boris_order, DepositTargets d, SpeciesCounters* cnt,
                                                  uint32_t* dead_bits, int injected_only) {
  using Acc = typename AccT<DET>::type;
  extern __shared__ __align__(16) unsigned char smem[];
  float* sEx = reinterpret_cast<float*>(smem);
  float* sEy = sEx + (PUSH ? kWin : 0);
  float* sBz = sEy + (PUSH ? kWin : 0);
  Acc* sRho = reinterpret_cast<Acc*>(smem + (PUSH ? (BZU ? 2 : 3) * size_t(kWin) * sizeof(float) : 0));
  Acc* sJx = sRho + kWin;
  Acc* sJy = sJx + kWin;
  __shared__ int s_red[4][kThreads / 32];
  __shared__ Window s_w;

  const uint32_t n = cnt->n;
  const uint32_t first = (!PUSH && injected_only) ? n - cnt->n_injected : 0u;
  const uint32_t base = first + blockIdx.x * uint32_t(kChunk);
  if (base >= n) return;  // uniform over the block
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int ngb = g.ngb;

  // ---- phase A: bounding box of the chunk's cells (re-read from L1 below)
  int mnx = INT_MAX, mny = INT_MAX, mxx = INT_MIN, mxy = INT_MIN;
#pragma unroll
  for (int i = 0; i < kPer; ++i) {
    const uint32_t k = base + uint32_t(i * kThreads + tid);
    const int32_t cl = k < n ? p.cell[k] : -1;
    if (cl >= 0) {
      const int ix = cell_ix(cl), iy = cell_iy(cl);
      if (interior(g, ix, iy)) {
        mnx = min(mnx, ix);
        mxx = max(mxx, ix);
        mny = min(mny, iy);
        mxy = max(mxy, iy);
      }
    }
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
    Window w;
    w.mnx = w.mny = INT_MAX;
    w.mxx = w.mxy = INT_MIN;
    for (int q = 0; q < kThreads / 32; ++q) {
      w.mnx = min(w.mnx, s_red[0][q]);
      w.mny = min(w.mny, s_red[1][q]);
      w.mxx = max(w.mxx, s_red[2][q]);
      w.mxy = max(w.mxy, s_red[3][q]);
    }
    w.use = 0;
    if (w.mnx != INT_MAX) {
      w.gx0 = w.mnx - ngb;
      w.gy0 = w.mny - ngb;
      w.gw = w.mxx - w.mnx + 2 + ORDER;
      w.gh = w.mxy - w.mny + 2 + ORDER;
      const int m = PUSH ? kMargin : 0;
      w.dx0 = w.gx0 - m;
      w.dy0 = w.gy0 - m;
      w.dw = w.gw + 2 * m;
      w.dh = w.gh + 2 * m;
      w.use = (w.dw * w.dh <= kWin) ? 1 : 0;
    }
    s_w = w;
  }
  __syncthreads();
  const Window w = s_w;

  // ---- phase B: stage the field window, clear the deposit window
  if (w.use) {
    if constexpr (PUSH) {
      const int nx = g.nx, ny = g.ny;
      for (int e = tid; e < w.gw * w.gh; e += kThreads) {
        const int col = w.gx0 + e % w.gw, row = w.gy0 + e / w.gw;
        sEx[e] = in_box(col, row, nx + 2, ny + 1) ? __ldg(f.Ex + col + row * (nx + 2)) : 0.0f;
        sEy[e] = in_box(col, row, nx + 1, ny + 2) ? __ldg(f.Ey + col + row * (nx + 1)) : 0.0f;
        if constexpr (!BZU) sBz[e] = in_box(col, row, nx + 2, ny + 2) ? __ldg(f.Bz + col + row * (nx + 2)) : 0.0f;
      }
    }
    if constexpr (DEP) {
      for (int e = tid; e < w.dw * w.dh; e += kThreads) {
        sRho[e] = Acc(0);
        if constexpr (CUR) {
          sJx[e] = Acc(0);
          sJy[e] = Acc(0);
        }
      }
    }
  }
  __syncthreads();

  // ---- phase C: particles
  uint32_t wcount[4] = {0, 0, 0, 0}, ninvalid = 0, ndead = 0, nslow = 0;
  double ke = 0.0;
#pragma unroll 1
  for (int i = 0; i < kPer; ++i) {
    const uint32_t k = base + uint32_t(i * kThreads + tid);
    int fl = 0;
    if (k < n) {
      const int32_t cell = p.cell[k];
      if (cell < 0) {
        fl = -cell;  // flagged before this push and not yet compacted: keep the flag
      } else {
        int ix = cell_ix(cell), iy = cell_iy(cell);
        float ox = p.ox[k], oy = p.oy[k];
        const bool inside = interior(g, ix, iy);
        if constexpr (!PUSH) {
          const Stagger sx = stagger(ix, ox), sy = stagger(iy, oy);
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
          if (inside && w.use)
            deposit_one<ORDER, DET, CUR, true, false>(g, w, sx, sy, wxn, wxh, wyn, wyh, c.scale, vx, vy, d, sRho, sJx, sJy);
          else if (inside)
            deposit_one<ORDER, DET, CUR, false, false>(g, w, sx, sy, wxn, wxh, wyn, wyh, c.scale, vx, vy, d, sRho, sJx, sJy);
          else
            deposit_one<ORDER, DET, CUR, false, true>(g, w, sx, sy, wxn, wxh, wyn, wyh, c.scale, vx, vy, d, sRho, sJx, sJy);
        } else {
          float vx = p.vx[k], vy = p.vy[k], vz = p.vz[k];
          const Stagger sx = stagger(ix, ox), sy = stagger(iy, oy);
          float wxn[ORDER + 1], wxh[ORDER + 1], wyn[ORDER + 1], wyh[ORDER + 1];
          shape<ORDER>(sx.hnode, wxn);
          shape<ORDER>(sx.hhalf, wxh);
          shape<ORDER>(sy.hnode, wyn);
          shape<ORDER>(sy.hhalf, wyh);
          float Epx = 0.0f, Epy = 0.0f, Bpz = 0.0f;
          if (inside && w.use)
            gather<ORDER, BZU, true, false>(g, f, w, sx, sy, wxn, wxh, wyn, wyh, sEx, sEy, sBz, Epx, Epy, Bpz);
          else if (inside)
            gather<ORDER, BZU, false, false>(g, f, w, sx, sy, wxn, wxh, wyn, wyh, sEx, sEy, sBz, Epx, Epy, Bpz);
          else
            gather<ORDER, BZU, false, true>(g, f, w, sx, sy, wxn, wxh, wyn, wyh, sEx, sEy, sBz, Epx, Epy, Bpz);
          if (!w.use) nslow++;
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
            // a live particle stays on the grid, or its next stencil would
            // leave the arrays (possible only for a displacement of more than
            // the domain in one step)
            if (fl == 0 && !interior(g, ix, iy)) fl = 5;
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
              const bool in_win = w.use && ix >= w.mnx - kMargin && ix <= w.mxx + kMargin &&
                                  iy >= w.mny - kMargin && iy <= w.mxy + kMargin;
              if (in_win)
                deposit_one<ORDER, DET, CUR, true, false>(g, w, nsx, nsy, wxn, wxh, wyn, wyh, c.scale, vx, vy, d,
                                                          sRho, sJx, sJy);
              else
                deposit_one<ORDER, DET, CUR, false, false>(g, w, nsx, nsy, wxn, wxh, wyn, wyh, c.scale, vx, vy, d,
                                                           sRho, sJx, sJy);
            }
          } else {
            p.cell[k] = -fl;
          }
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
    if constexpr (PUSH) {
      const uint32_t wbase = base + uint32_t(i * kThreads + wid * 32);
      const uint32_t bits = __ballot_sync(0xffffffffu, fl != 0);
      if (lane == 0 && wbase < n) dead_bits[wbase >> 5] = bits;
    }
  }

  // ---- phase D: flush the deposit window
  if constexpr (DEP) {
    __syncthreads();
    if (w.use) {
      const int nx = g.nx, ny = g.ny;
      for (int e = tid; e < w.dw * w.dh; e += kThreads) {
        const int col = w.dx0 + e % w.dw, row = w.dy0 + e / w.dw;
        const Acc r = sRho[e];
        if (r != Acc(0) && in_box(col, row, nx + 1, ny + 1)) {
          if constexpr (DET)
            gadd(d.acc_rho + col + row * (nx + 1), r);
          else
            gadd(d.f64_rho + col + row * (nx + 1), r);
        }
        if constexpr (CUR) {
          const Acc a = sJx[e], b = sJy[e];
          if (a != Acc(0) && in_box(col, row, nx + 2, ny + 1)) {
            if constexpr (DET)
              gadd(d.acc_jx + col + row * (nx + 2), a);
            else
              gadd(d.f64_jx + col + row * (nx + 2), a);
          }
          if (b != Acc(0) && in_box(col, row, nx + 1, ny + 2)) {
            if constexpr (DET)
              gadd(d.acc_jy + col + row * (nx + 1), b);
            else
              gadd(d.f64_jy + col + row * (nx + 1), b);
          }
        }
      }
    }
  }

  if constexpr (PUSH) {
    const uint32_t s_dead = warp_sum(ndead);
    const uint32_t s_w0 = warp_sum(wcount[0]), s_w1 = warp_sum(wcount[1]);
    const uint32_t s_w2 = warp_sum(wcount[2]), s_w3 = warp_sum(wcount[3]);
    const uint32_t s_inv = warp_sum(ninvalid), s_slow = warp_sum(nslow);
    const double s_ke = warp_sum(ke);
    if (lane == 0) {
      if (s_dead) atomicAdd(&cnt->n_dead, s_dead);
      if (s_w0) atomicAdd(&cnt->wall[0], s_w0);
      if (s_w1) atomicAdd(&cnt->wall[1], s_w1);
      if (s_w2) atomicAdd(&cnt->wall[2], s_w2);
      if (s_w3) atomicAdd(&cnt->wall[3], s_w3);
      if (s_inv) atomicAdd(&cnt->invalid, s_inv);
      if (s_slow) atomicAdd(&cnt->n_slow, s_slow);
      if (s_ke != 0.0) atomicAdd(&cnt->ke, s_ke);
    }
  }
}

template <int ORDER, bool PUSH, bool DEP, bool DET, bool CUR, bool BZU>
void launch_pic(uint32_t nblocks, cudaStream_t s, GridDims g, ParticleArrays p, FieldPtrs f, PushConsts c, int boris,
                DepositTargets d, SpeciesCounters* cnt, uint32_t* bits, int injected_only) {
  auto kern = k_pic<ORDER, PUSH, DEP, DET, CUR, BZU>;
  constexpr size_t bytes = smem_bytes<ORDER, PUSH, DEP, DET, BZU>(CUR);
  static bool configured = false;
  if (!configured) {
    GP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
    configured = true;
  }
  kern<<<nblocks, kThreads, bytes, s>>>(g, p, f, c, boris, d, cnt, bits, injected_only);
}

template <int ORDER, bool PUSH>
void dispatch_pic(bool dep, bool det, bool cur, bool bzu, uint32_t nblocks, cudaStream_t s, GridDims g,
                  ParticleArrays p, FieldPtrs f, PushConsts c, int boris, DepositTargets d, SpeciesCounters* cnt,
                  uint32_t* bits, int injected_only) {
  // PUSH=false always deposits; Bz is not read then.
#define GP_PIC(DEP, DET, CUR, BZU) \
  launch_pic<ORDER, PUSH, DEP, DET, CUR, BZU>(nblocks, s, g, p, f, c, boris, d, cnt, bits, injected_only)
  if constexpr (PUSH) {
    if (!dep) {
      bzu ? GP_PIC(false, false, false, true) : GP_PIC(false, false, false, false);
    } else if (det) {
      if (cur)
        bzu ? GP_PIC(true, true, true, true) : GP_PIC(true, true, true, false);
      else
        bzu ? GP_PIC(true, true, false, true) : GP_PIC(true, true, false, false);
    } else {
      if (cur)
        bzu ? GP_PIC(true, false, true, true) : GP_PIC(true, false, true, false);
      else
        bzu ? GP_PIC(true, false, false, true) : GP_PIC(true, false, false, false);
    }
  } else {
    if (det)
      cur ? GP_PIC(true, true, true, true) : GP_PIC(true, true, false, true);
    else
      cur ? GP_PIC(true, false, true, true) : GP_PIC(true, false, false, true);
  }
#undef GP_PIC
}

// ------------------------------------------------------------- tile sort
constexpr int kSortThreads = 256;
constexpr int kSortPer = 16;
constexpr int kSortChunk = kSortThreads * kSortPer;

__device__ __forceinline__ int tile_bin(int32_t cell, int tile, int ntx, int nbins) {
  if (cell < 0) return nbins;  // flagged particles (none after compaction) go last
  return (cell_iy(cell) / tile) * ntx + cell_ix(cell) / tile;
}

__global__ void __launch_bounds__(kSortThreads) k_sort_hist(const int32_t* cell, const SpeciesCounters* cnt, int tile,
                                                            int ntx, int nbins, uint32_t* bins) {
  extern __shared__ uint32_t sh[];
  const uint32_t n = cnt->n;
  const uint32_t base = blockIdx.x * uint32_t(kSortChunk);
  if (base >= n) return;
  for (int b = threadIdx.x; b <= nbins; b += kSortThreads) sh[b] = 0;
  __syncthreads();
  for (int i = 0; i < kSortPer; ++i) {
    const uint32_t k = base + uint32_t(i * kSortThreads) + threadIdx.x;
    if (k < n) atomicAdd(&sh[tile_bin(cell[k], tile, ntx, nbins)], 1u);
  }
  __syncthreads();
  for (int b = threadIdx.x; b <= nbins; b += kSortThreads)
    if (sh[b]) atomicAdd(&bins[b], sh[b]);
}

__global__ void __launch_bounds__(1024) k_sort_scan(const uint32_t* bins, uint32_t* offsets, int nb) {
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_base;
  if (threadIdx.x == 0) s_base = 0;
  __syncthreads();
  for (int b0 = 0; b0 < nb; b0 += blockDim.x) {
    const int b = b0 + threadIdx.x;
    const uint32_t c = b < nb ? bins[b] : 0u;
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
    if (b < nb) offsets[b] = s_base + s_warp[wid] + incl - c;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) s_base += s_warp[wid] + incl;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kSortThreads) k_sort_scatter(ParticleArrays src, ParticleArrays dst,
                                                               const SpeciesCounters* cnt, int tile, int ntx, int nbins,
                                                               uint32_t* offsets) {
  extern __shared__ uint32_t sh[];
  uint32_t* cntb = sh;              // nbins + 1
  uint32_t* baseb = sh + nbins + 1;  // nbins + 1
  const uint32_t n = cnt->n;
  const uint32_t base = blockIdx.x * uint32_t(kSortChunk);
  if (base >= n) return;
  for (int b = threadIdx.x; b <= nbins; b += kSortThreads) cntb[b] = 0;
  __syncthreads();
  int bin[kSortPer];
#pragma unroll
  for (int i = 0; i < kSortPer; ++i) {
    const uint32_t k = base + uint32_t(i * kSortThreads) + threadIdx.x;
    bin[i] = k < n ? tile_bin(src.cell[k], tile, ntx, nbins) : -1;
    if (bin[i] >= 0) atomicAdd(&cntb[bin[i]], 1u);
  }
  __syncthreads();
  for (int b = threadIdx.x; b <= nbins; b += kSortThreads) {
    const uint32_t c = cntb[b];
    baseb[b] = c ? atomicAdd(&offsets[b], c) : 0u;
    cntb[b] = 0;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kSortPer; ++i) {
    if (bin[i] < 0) continue;
    const uint32_t k = base + uint32_t(i * kSortThreads) + threadIdx.x;
    const uint32_t dpos = baseb[bin[i]] + atomicAdd(&cntb[bin[i]], 1u);
    dst.cell[dpos] = src.cell[k];
    dst.ox[dpos] = src.ox[k];
    dst.oy[dpos] = src.oy[k];
    dst.vx[dpos] = src.vx[k];
    dst.vy[dpos] = src.vy[k];
    dst.vz[dpos] = src.vz[k];
  }
}

}  // namespace

void push(int order, int boris_order, bool dep, bool det, bool cur, bool bzu, GridDims g, ParticleArrays p,
          FieldPtrs f, PushConsts c, DepositTargets d, SpeciesCounters* cnt, uint32_t* dead_bits, uint32_t n_bound,
          cudaStream_t s) {
  // Zero the per-push counters (everything after n).
  GP_CUDA(cudaMemsetAsync(&cnt->n_dead, 0, sizeof(SpeciesCounters) - offsetof(SpeciesCounters, n_dead), s));
  if (n_bound == 0) return;
  const uint32_t nblocks = (n_bound + kChunk - 1) / kChunk;
  switch (order) {
    case 1: dispatch_pic<1, true>(dep, det, cur, bzu, nblocks, s, g, p, f, c, boris_order, d, cnt, dead_bits, 0); break;
    case 3: dispatch_pic<3, true>(dep, det, cur, bzu, nblocks, s, g, p, f, c, boris_order, d, cnt, dead_bits, 0); break;
    case 5: dispatch_pic<5, true>(dep, det, cur, bzu, nblocks, s, g, p, f, c, boris_order, d, cnt, dead_bits, 0); break;
    default: throw std::invalid_argument("WeightingOrder must be 1, 3 or 5");
  }
  GP_LAUNCH_CHECK();
}

void deposit(int order, bool det, bool cur, GridDims g, ParticleArrays p, float scale, DepositTargets d,
             const SpeciesCounters* cnt, uint32_t n_bound, bool injected_only, cudaStream_t s) {
  if (n_bound == 0) return;
  const uint32_t nblocks = (n_bound + kChunk - 1) / kChunk;
  PushConsts c{};
  c.scale = scale;
  FieldPtrs f{nullptr, nullptr, nullptr};
  auto* mc = const_cast<SpeciesCounters*>(cnt);
  const int inj = injected_only ? 1 : 0;
  switch (order) {
    case 1: dispatch_pic<1, false>(true, det, cur, true, nblocks, s, g, p, f, c, 2, d, mc, nullptr, inj); break;
    case 3: dispatch_pic<3, false>(true, det, cur, true, nblocks, s, g, p, f, c, 2, d, mc, nullptr, inj); break;
    case 5: dispatch_pic<5, false>(true, det, cur, true, nblocks, s, g, p, f, c, 2, d, mc, nullptr, inj); break;
    default: throw std::invalid_argument("WeightingOrder must be 1, 3 or 5");
  }
  GP_LAUNCH_CHECK();
}

int sort_bins(GridDims g, int tile) { return ((g.nx + tile) / tile) * ((g.ny + tile) / tile); }

int sort_tile_size(GridDims g) {
  int t = 8;
  while (sort_bins(g, t) > 8192) t *= 2;
  return t;
}

void sort_by_tile(GridDims g, int tile, ParticleArrays src, ParticleArrays dst, const SpeciesCounters* cnt,
                  uint32_t* bins, uint32_t* offsets, uint32_t n_bound, cudaStream_t s) {
  if (n_bound == 0) return;
  const int ntx = (g.nx + tile) / tile;
  const int nbins = sort_bins(g, tile);
  const uint32_t nblocks = (n_bound + kSortChunk - 1) / kSortChunk;
  static bool configured = false;
  if (!configured) {  // up to 2 x 8193 bins of shared memory
    GP_CUDA(cudaFuncSetAttribute(k_sort_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, 8193 * 4));
    GP_CUDA(cudaFuncSetAttribute(k_sort_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * 8193 * 4));
    configured = true;
  }
  if (nbins > 8192) throw std::invalid_argument("sort tile too small for the grid");
  GP_CUDA(cudaMemsetAsync(bins, 0, size_t(nbins + 1) * sizeof(uint32_t), s));
  k_sort_hist<<<nblocks, kSortThreads, size_t(nbins + 1) * sizeof(uint32_t), s>>>(src.cell, cnt, tile, ntx, nbins,
                                                                                  bins);
  GP_LAUNCH_CHECK();
  k_sort_scan<<<1, 1024, 0, s>>>(bins, offsets, nbins + 1);
  GP_LAUNCH_CHECK();
  k_sort_scatter<<<nblocks, kSortThreads, 2 * size_t(nbins + 1) * sizeof(uint32_t), s>>>(src, dst, cnt, tile, ntx,
                                                                                         nbins, offsets);
  GP_LAUNCH_CHECK();
}

}  // namespace kern
}  // namespace gample
