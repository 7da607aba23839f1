// particle_kernels.cu -- per-particle kernels of the PIC step (sm_100a).
//
//  k_pic<PUSH=true>   gather (order 1/3/5 B-splines on the staggered grid) +
//                     Boris rotation (order 2/4/6) + position update +
//                     boundary conditions (src/Particle.mm:65-278), optionally
//                     fused with the charge/current deposit of the new
//                     positions (src/Particle.mm:281-389).
//  k_pic<PUSH=false>  deposit of the current positions (src/Particle.mm:281-389).
//
// Work decomposition: one CTA per chunk of kChunk consecutive particles.
// Because the particles are cell-sorted, a chunk covers a small box of cells;
// the CTA stages the field window of that box (Ex, Ey, Bz) in shared memory
// and accumulates its deposit in a shared-memory window that is flushed with
// one global atomic per touched node (FP64 per species, or exact int64 in the
// deterministic mode). Chunks whose box does not fit (unsorted or drifted
// particles) fall back to direct global gathers/atomics, per chunk; particles
// not strictly inside the grid use bounds-checked stencils.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdio>
#include <mutex>
#include <type_traits>

#include "device.hpp"
#include "kernels.hpp"
#include "pic_common.cuh"

namespace gample {
namespace kern {

namespace {

constexpr int kThreads = 256;
constexpr int kPer = kPushChunkPer;          // particles per thread
constexpr int kChunk = kThreads * kPer;      // particles per CTA
constexpr int kWin = 1600;                   // entries of a shared-memory window (e.g. 40 x 40)
constexpr int kMargin = 2;                   // deposit-window margin for the motion of one step (cells)
constexpr int kReach = 12;                   // window box: cells within kReach of the chunk's middle particle
constexpr size_t kDepositBudget = 98304;     // shared-memory bytes for the deposit window copies
constexpr int kPW = 20;                      // row stride of a lane-private deposit window (entries)
constexpr int kPrivWords = 10752;            // words for 32 lane-private windows (42 KB)
// Gather tables: one polynomial (4 float4 of coefficients) per entry, entries
// 5 float4 apart and rows padded to 2 mod 8 float4, so that a 16-byte load of
// entry (col, row) falls in bank group (5 col + 2 row + const) mod 8 and the 8
// lanes served together by a 16-byte shared load, whose particles lie in
// neighbouring cells, mostly use distinct banks.
constexpr int kTabEntry = 5;                                // float4 per polynomial
constexpr int kTabFloat4 = 2 * kWin / 4;                    // float4 that fit in the Ex/Ey windows
__host__ __device__ constexpr int tab_row_stride(int entries) {
  return entries * kTabEntry + ((2 - entries * kTabEntry) & 7);
}

__device__ __forceinline__ uint32_t warp_sum(uint32_t v) { return __reduce_add_sync(0xffffffffu, v); }
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ bool in_box(int i, int j, int w, int h) { return i >= 0 && j >= 0 && i < w && j < h; }

// ---- field staging by bulk tensor copies (TMA). One mbarrier per CTA, used
// once (phase 0): thread 0 arms it with the byte count and issues the copies
// of the Ex and Ey tiles; every thread waits on it, with a bounded number of
// polls, before reading the tiles.
static_assert(kFieldBoxes == 3 && kFieldBoxW[0] == 20 && kFieldBoxH[0] == 8 && kFieldBoxW[1] == 24 &&
                  kFieldBoxH[1] == 16 && kFieldBoxW[2] == 40 && kFieldBoxH[2] == 40,
              "box table of field_box()");
// Smallest box that covers need_w x need_h, or -1.
__device__ __forceinline__ int field_box(int need_w, int need_h) {
  if (need_w <= 20 && need_h <= 8) return 0;
  if (need_w <= 24 && need_h <= 16) return 1;
  if (need_w <= 40 && need_h <= 40) return 2;
  return -1;
}
__device__ __forceinline__ int field_box_w(int b) { return b == 0 ? 20 : (b == 1 ? 24 : 40); }
__device__ __forceinline__ int field_box_h(int b) { return b == 0 ? 8 : (b == 1 ? 16 : 40); }
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ void mbar_init1(uint32_t bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// Tile (x, y) .. (x + box w - 1, y + box h - 1) of a 2D tensor map into
// shared memory at dst (row stride = box width); x is a multiple of 4
// elements (16 bytes), dst 128-byte aligned.
__device__ __forceinline__ void tma_tile(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}
__device__ __forceinline__ bool mbar_wait0(uint32_t bar) {
  for (int i = 0; i < (1 << 20); ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar)
        : "memory");
    if (done) return true;
  }
  return false;
}

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
  int ds;                // deposit window row stride (>= dw, congruent to ORDER + 1 mod 32)
  int priv;              // 1: 32 lane-private deposit windows, row stride kPW
  int ps;                // their copy stride (odd, >= kPW * dh)
  int tab;               // 1: gather table of the box's cells instead of the field windows
  int tbw, tbh;          // box size in cells
  int xrs, yrs, yoff;    // Ex / Ey table row strides and the Ey table's start (float4)
  // staged Ex / Ey tiles: origin, row stride and rows (gather windows: the
  // window itself, or the TMA box that covers it; tables: the box the table
  // build reads); tma: 1 when a bulk tensor copy stages them, into sEx / sEy
  // (windows) or at byte soff of sEx, Ey one box further (tables)
  int sx0, sy0, sstr, shh;
  int tma, sbox, soff;
};

// r[t] = w[(t + sh) mod N] for a per-lane shift sh in [0, N).
template <int N>
__device__ __forceinline__ void rotate(const float (&w)[N], int sh, float (&r)[N]) {
#pragma unroll
  for (int t = 0; t < N; ++t) {
    float v = w[t];
#pragma unroll
    for (int q = 1; q < N; ++q)
      if (sh == q) v = w[(t + q) % N];
    r[t] = v;
  }
}

// Deposit one particle's weights. WIN: into the shared-memory window;
// otherwise global (CHECKED skips nodes outside the arrays, which carry
// weight zero for a particle exactly on the far wall, src/Particle.mm:357-373).
//
// In the window each lane visits the (ORDER+1)^2 stencil nodes in its own
// rotated order: lane L starts at node (L mod N, (L / N) mod N). Lanes of a
// warp mostly share a cell (the particles are cell-sorted), so without the
// rotation all 32 lanes would add to the same address at every step; with it
// the first N^2 lanes add to distinct nodes, and the window row stride
// (congruent to N mod 32) puts those nodes in distinct banks. The summands
// are the same as in the unrotated loop; only their order of arrival differs.
// |v / c| < 1 in FP32 for both components (always true without currents).
template <bool CUR>
__device__ __forceinline__ bool sublight(float vx, float vy) {
  if constexpr (CUR) {
    constexpr float inv_c = float(1.0 / 2.99792458e10);
    return fabsf(__fmul_rn(vx, inv_c)) < 1.0f && fabsf(__fmul_rn(vy, inv_c)) < 1.0f;
  } else {
    return true;
  }
}

__device__ __forceinline__ long long wsum(const int* s, int ihi, int ilo) {
  return (static_cast<long long>(s[ihi]) << 20) + static_cast<long long>(static_cast<unsigned>(s[ilo]));
}

// Deposit windows: each array has kCopies private copies, lane L adding into
// copy (L / N^2) mod kCopies. With the rotated stencil order this gives the
// 32 lanes of a warp whose particles share a cell 32 distinct addresses: N^2
// distinct nodes per copy, and the copy stride (congruent to N^2 mod 32)
// moves each copy onto its own banks. Copies are summed at the flush.
//
// Two number formats. The deterministic mode, and any deposit with currents,
// holds exact 2^-40 fixed-point sums in two words per node (below). The atomic
// mode without currents holds one 32-bit word per node with the weight
// quantised to 2^-kQBits (2^-22 for orders 1 and 3, 2^-21 for order 5): the
// rounding of a contribution is at most 2^-(kQBits+1) in weight units, finer
// than the FP32 atomic additions of the reference's deposit (each rounds the
// running node sum to 24 bits, src/Particle.mm:362), and the window sums stay
// exact integers, so only the FP64 flush order varies between runs.
template <int ORDER, bool CUR, bool DET>
struct DepositLayout {
  static constexpr int kN2 = (ORDER + 1) * (ORDER + 1);
  static constexpr int kStride = kWin + kN2 % 32;
  static constexpr bool kSingle = !DET && !CUR;
  static constexpr int kQBits = ORDER == 5 ? 21 : 22;
  static constexpr int kArrays = kSingle ? 1 : (CUR ? 6 : 2);  // words of rho (jx, jy)
  static constexpr size_t kCopyBytes = size_t(kStride) * kArrays * sizeof(int);
  static constexpr int copies() {
    int c = kN2 >= 32 ? 1 : 32 / kN2;
    while (c > 1 && size_t(c) * kCopyBytes > kDepositBudget) c >>= 1;
    return c;
  }
  static constexpr int kCopies = copies();
  static constexpr int kArrayBytes = kCopies * kStride * int(sizeof(int));  // one array, all copies
  static constexpr size_t kSharedBytes = size_t(kCopies) * kCopyBytes;
  // the single-word layout may also hold 32 lane-private windows (kPrivWords)
  static constexpr size_t kBytes =
      kSingle && size_t(kPrivWords) * sizeof(int) > kSharedBytes ? size_t(kPrivWords) * sizeof(int) : kSharedBytes;
  // single word: a copy receives at most kChunk / kCopies contributions per
  // node, each at most the largest stencil weight (1, (2/3)^2, (11/20)^2)
  static constexpr double kMaxW = ORDER == 1 ? 1.0 : (ORDER == 3 ? 0.4445 : 0.3026);
  static_assert(!kSingle || double(kChunk / kCopies) * kMaxW * double(1 << kQBits) < 2147483647.0,
                "single-word deposit window could overflow");
  // lane-private windows: copy L takes lane L of every warp, kPer particles
  // each, so at most kPer * (kThreads / 32) contributions per node and word
  static_assert(!kSingle || double(kPer) * (kThreads / 32) * kMaxW * double(1 << kQBits) < 2147483647.0,
                "a lane-private window word could overflow");
  // the flush's sum of the 32 lane-private copies fits 32 unsigned bits
  static constexpr bool kPrivSum32 = 32.0 * kPer * (kThreads / 32) * kMaxW * double(1 << kQBits) < 4294967295.0;
};

// This lane's copy of the window arrays: shared-memory byte address of its rho
// hi-word copy; array a (rho hi, rho lo, jx hi, jx lo, jy hi, jy lo) lies
// a * kArrayBytes further.
struct WinPtrs {
  uint32_t rho;
};

// Shared-memory windows hold exact fixed-point sums (weights quantised to
// 2^-40) split over two 32-bit words per node: hi = q >> 20 (signed) and
// lo = q & (2^20 - 1), each added with a native 32-bit integer reduction (the
// floating-point and 64-bit shared-memory atomics are compare-and-swap
// loops that retry under contention). A copy of a window receives at most
// kChunk contributions per node, each with |q| <= 2^40, so neither word can
// overflow; the flush recombines hi * 2^20 + lo in 64 bits.
// One contribution: hi word at addr + HI, lo word at addr + LO (byte offsets
// known at compile time, folded into the instructions).
template <int HI, int LO>
__device__ __forceinline__ void wadd_s(uint32_t addr, long long q) {
  asm volatile("red.shared.add.s32 [%0+%1], %2;" ::"r"(addr), "n"(HI), "r"(int(q >> 20)) : "memory");
  asm volatile("red.shared.add.s32 [%0+%1], %2;" ::"r"(addr), "n"(LO), "r"(int(q & 0xFFFFF)) : "memory");
}

// The integers nearest to x0 * y and x1 * y (0 <= x * y <= 2^22), each
// rounded once: fma(x, y, 1.5 * 2^23) holds it in the low mantissa bits (the
// ulp at 1.5 * 2^23 is 1), read off by subtracting the bits of 1.5 * 2^23.
__device__ __forceinline__ int2 fixed_pair(float x0, float x1, float y) {
  constexpr float kMagic = 12582912.0f;    // 1.5 * 2^23
  constexpr int kMagicBits = 0x4B400000;  // its bit pattern
  const float2 r = __ffma2_rn(make_float2(x0, x1), make_float2(y, y), make_float2(kMagic, kMagic));
  return make_int2(__float_as_int(r.x) - kMagicBits, __float_as_int(r.y) - kMagicBits);
}

// The window path accumulates quant40(w) for rho and quant40(w * v / c) for
// the currents (rn(w * 2^kQBits) for rho in the single-word layout); the
// caller sends a particle with |v| >= c (|w v / c| could exceed 1) to the
// global path instead.
template <int ORDER, bool DET, bool CUR, bool WIN, bool CHECKED>
__device__ __forceinline__ void deposit_one(const GridDims& g, const Window& w, int lane, const Stagger& sx,
                                            const Stagger& sy, const float (&wxn)[ORDER + 1],
                                            const float (&wxh)[ORDER + 1], const float (&wyn)[ORDER + 1],
                                            const float (&wyh)[ORDER + 1], float scale, float vx, float vy,
                                            const DepositTargets& d, const WinPtrs& s) {
  using C = Contrib<DET>;
  constexpr int N = ORDER + 1;
  constexpr float inv_c = float(1.0 / 2.99792458e10);
  const int ngb = g.ngb, nx = g.nx, ny = g.ny;
  const int rc = sx.node - ngb, rr = sy.node - ngb;  // rho / jy column base, rho / jx row base
  const int xc = sx.half - ngb + 1, yr = sy.half - ngb + 1;  // jx column base, jy row base
  if constexpr (WIN) {
    using DL = DepositLayout<ORDER, CUR, DET>;
    constexpr int kA = DL::kArrayBytes;
    // x weights pre-scaled by the fixed-point unit (exact): quant(wx * wy) == rn(wx' * wy)
    constexpr float kUnit = DL::kSingle ? float(1 << DL::kQBits) : kQuant;
    const int si = lane % N, sj = (lane / N) % N;
    float rxn[N], ryn[N];
    rotate<N>(wxn, si, rxn);
    rotate<N>(wyn, sj, ryn);
#pragma unroll
    for (int t = 0; t < N; ++t) rxn[t] = __fmul_rn(rxn[t], kUnit);
    uint32_t col[N], row[N];  // byte offsets of the rotated stencil columns / rows
    const uint32_t ds4 = 4u * uint32_t(w.ds);
#pragma unroll
    for (int t = 0; t < N; ++t) {
      constexpr bool kPow2 = (N & (N - 1)) == 0;
      const int cs = kPow2 ? ((t + si) & (N - 1)) : (t + si >= N ? t + si - N : t + si);
      const int rs = kPow2 ? ((t + sj) & (N - 1)) : (t + sj >= N ? t + sj - N : t + sj);
      col[t] = 4u * uint32_t(cs);
      row[t] = uint32_t(rs) * ds4;
    }
    const uint32_t arho = s.rho + 4u * uint32_t((rc - w.dx0) + (rr - w.dy0) * w.ds);
#pragma unroll
    for (int a = 0; a < N; ++a)
#pragma unroll
      for (int b = 0; b < N; ++b) {
        if constexpr (DL::kSingle) {
          if (b % 2 == 0) {  // rounded once, two nodes per packed FFMA2 (as in priv_add)
            const int2 q = fixed_pair(rxn[b], rxn[b + 1], ryn[a]);
            asm volatile("red.shared.add.s32 [%0], %1;" ::"r"(arho + col[b] + row[a]), "r"(q.x) : "memory");
            asm volatile("red.shared.add.s32 [%0], %1;" ::"r"(arho + col[b + 1] + row[a]), "r"(q.y) : "memory");
          }
        } else {
          wadd_s<0, kA>(arho + col[b] + row[a], __float2ll_rn(__fmul_rn(rxn[b], ryn[a])));
        }
      }
    if constexpr (CUR) {
      float rxh[N], ryh[N];
      rotate<N>(wxh, si, rxh);
      rotate<N>(wyh, sj, ryh);
#pragma unroll
      for (int t = 0; t < N; ++t) rxh[t] = __fmul_rn(rxh[t], kQuant);
      const float ux = __fmul_rn(vx, inv_c), uy = __fmul_rn(vy, inv_c);
      const uint32_t ajx = s.rho + 4u * uint32_t((xc - w.dx0) + (rr - w.dy0) * w.ds);
      const uint32_t ajy = s.rho + 4u * uint32_t((rc - w.dx0) + (yr - w.dy0) * w.ds);
#pragma unroll
      for (int a = 0; a < N; ++a)
#pragma unroll
        for (int b = 0; b < N; ++b) {
          wadd_s<2 * kA, 3 * kA>(ajx + col[b] + row[a], __float2ll_rn(__fmul_rn(__fmul_rn(rxh[b], ryn[a]), ux)));
          wadd_s<4 * kA, 5 * kA>(ajy + col[b] + row[a], __float2ll_rn(__fmul_rn(__fmul_rn(rxn[b], ryh[a]), uy)));
        }
    }
  } else {
#pragma unroll
    for (int i = 0; i <= ORDER; ++i)
#pragma unroll
      for (int j = 0; j <= ORDER; ++j) {
        const auto v = C::rho(__fmul_rn(wxn[i], wyn[j]), scale);
        if (CHECKED && !in_box(rc + i, rr + j, nx + 1, ny + 1)) continue;
        if constexpr (DET)
          gadd(d.acc_rho + (rc + i) + (rr + j) * (nx + 1), v);
        else
          gadd(d.f64_rho + (rc + i) + (rr + j) * (nx + 1), v);
      }
    if constexpr (CUR) {
      const float ux = __fmul_rn(vx, inv_c), uy = __fmul_rn(vy, inv_c);
#pragma unroll
      for (int i = 0; i <= ORDER; ++i)
#pragma unroll
        for (int j = 0; j <= ORDER; ++j) {
          const auto a = C::cur(__fmul_rn(wxh[i], wyn[j]), scale, vx, ux);
          const auto b = C::cur(__fmul_rn(wxn[i], wyh[j]), scale, vy, uy);
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

// Lane-private single-word windows: when 32 copies of a small deposit window
// fit, lane L adds into its own copy at L * ps words (ps odd, so lanes adding
// to the same node of their copies hit 32 distinct banks). No stencil
// rotation is needed, and every node offset is a compile-time immediate of
// the row stride kPW. Lane L of every warp shares copy L, so a copy receives
// at most kPer * (kThreads / 32) contributions per node.
// Each contribution is the integer nearest to wx * 2^kQBits * wy, rounded once
// (fixed_pair: two x-neighbouring nodes per packed FFMA2), as in the rotated
// shared layout, so the integer window sums of the two layouts are the same.
template <int N, int K = 0>
__device__ __forceinline__ void priv_add(uint32_t a0, const float (&rx)[N], const float (&ry)[N]) {
  static_assert(N % 2 == 0, "nodes are taken in x pairs");
  if constexpr (K < N * N) {
    const int2 q = fixed_pair(rx[K % N], rx[K % N + 1], ry[K / N]);
    asm volatile("red.shared.add.s32 [%0+%1], %2;" ::"r"(a0), "n"(4 * (K % N + (K / N) * kPW)), "r"(q.x)
                 : "memory");
    asm volatile("red.shared.add.s32 [%0+%1], %2;" ::"r"(a0), "n"(4 * (K % N + 1 + (K / N) * kPW)), "r"(q.y)
                 : "memory");
    priv_add<N, K + 2>(a0, rx, ry);
  }
}

template <int ORDER>
__device__ __forceinline__ void deposit_priv(const Window& w, uint32_t lane_base, int ngb, const Stagger& sx,
                                             const Stagger& sy, const float (&wxn)[ORDER + 1],
                                             const float (&wyn)[ORDER + 1]) {
  constexpr int N = ORDER + 1;
  constexpr float kUnit = float(1 << DepositLayout<ORDER, false, false>::kQBits);
  float rx[N];
#pragma unroll
  for (int t = 0; t < N; ++t) rx[t] = __fmul_rn(wxn[t], kUnit);
  const uint32_t a0 = lane_base + 4u * uint32_t((sx.node - ngb - w.dx0) + (sy.node - ngb - w.dy0) * kPW);
  priv_add<N>(a0, rx, wyn);
}

// Gather table (order 3, uniform Bz). Inside one cell, for a fixed choice of
// the half-shifted stencil (offset below or above 1/2), the gathered field is
// a bicubic polynomial of the particle's offsets: Ex(hx, oy) with hx the
// half-shifted x offset and Ey(ox, hy). An Ex polynomial belongs to a
// half-shifted column (the upper half of one cell and the lower half of the
// next) and a row, an Ey polynomial to a column and a half-shifted row. The
// CTA tabulates the monomial coefficients of every polynomial its box needs,
//   C[n][m] = sum_i sum_j A[i][m] A[j][n] F(tap i, tap j),
// with A[i][m] the coefficient of h^m in the cubic B-spline weight of tap i
// (shape<3>), and a particle evaluates its two polynomials by Horner's rule:
// 8 shared 16-byte loads and 30 multiply-adds instead of four weight vectors,
// 32 loads and 40 multiply-adds. The sums equal the stencil sums up to FP32
// rounding.
__device__ __forceinline__ float cubic_coef(int tap, int m) {
  // rows: taps 0..3; columns: powers h^0..h^3 of shape<3>'s weights
  constexpr float kA[4][4] = {{1.0f / 6.0f, -0.5f, 0.5f, -1.0f / 6.0f},
                              {2.0f / 3.0f, 0.0f, -1.0f, 0.5f},
                              {1.0f / 6.0f, 0.5f, 0.5f, -0.5f},
                              {0.0f, 0.0f, 0.0f, 1.0f / 6.0f}};
  return kA[tap][m];
}

// Coefficients of one polynomial from its 4 x 4 taps F[i + 4 j] (i: column
// tap, j: row tap), stored by power of h: c[m] = (C[0][m], C[1][m], C[2][m],
// C[3][m]), so that one 16-byte load holds the coefficient of h^m of all four
// powers of k and the four Horner chains in h run as two packed pairs.
__device__ __forceinline__ void tab_build(const float (&F)[16], float4* c) {
  float T[4][4];  // T[i][n] = sum_j F(i, j) A[j][n]
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      float t = 0.0f;
#pragma unroll
      for (int j = 0; j < 4; ++j) t = fmaf(F[i + 4 * j], cubic_coef(j, n), t);
      T[i][n] = t;
    }
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    float r[4];
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      float t = 0.0f;
#pragma unroll
      for (int i = 0; i < 4; ++i) t = fmaf(cubic_coef(i, m), T[i][n], t);
      r[n] = t;
    }
    c[m] = make_float4(r[0], r[1], r[2], r[3]);
  }
}

// sum_n k^n sum_m C[n][m] h^m: p_n = ((C[n][3] h + C[n][2]) h + C[n][1]) h +
// C[n][0] for n = 0, 1 and n = 2, 3 as packed FP32 pairs (sm_100 FFMA2; each
// half rounds exactly like the scalar fused multiply-add), then Horner in k.
__device__ __forceinline__ float tab_eval(const float4* c, float h, float k) {
  const float4 c0 = c[0], c1 = c[1], c2 = c[2], c3 = c[3];
  const float2 hh = make_float2(h, h);
  float2 p01 = make_float2(c3.x, c3.y), p23 = make_float2(c3.z, c3.w);
  p01 = __ffma2_rn(p01, hh, make_float2(c2.x, c2.y));
  p23 = __ffma2_rn(p23, hh, make_float2(c2.z, c2.w));
  p01 = __ffma2_rn(p01, hh, make_float2(c1.x, c1.y));
  p23 = __ffma2_rn(p23, hh, make_float2(c1.z, c1.w));
  p01 = __ffma2_rn(p01, hh, make_float2(c0.x, c0.y));
  p23 = __ffma2_rn(p23, hh, make_float2(c0.z, c0.w));
  return fmaf(fmaf(fmaf(p23.y, k, p23.x), k, p01.y), k, p01.x);
}

// Gather Ex, Ey (and Bz) for one particle (src/Particle.mm:142-154).
// WIN: from the staged windows; CHECKED: global with bounds checks (a tap
// outside the arrays contributes zero). Every path evaluates the same
// separable sum -- each stencil row reduced with the x weights, then the row
// sums with the y weights (20 instead of 32 multiply-adds per component) --
// so a particle's result does not depend on which path its chunk takes (the
// gather tables of the atomic mode excepted: they agree to FP32 rounding).
template <int ORDER, bool BZU, bool WIN, bool CHECKED>
__device__ __forceinline__ void gather(const GridDims& g, const FieldPtrs& f, const Window& w, const Stagger& sx,
                                       const Stagger& sy, const float (&wxn)[ORDER + 1],
                                       const float (&wxh)[ORDER + 1], const float (&wyn)[ORDER + 1],
                                       const float (&wyh)[ORDER + 1], const float* sEx, const float* sEy,
                                       const float* sBz, float& Epx, float& Epy, float& Bpz) {
  const int ngb = g.ngb, nx = g.nx, ny = g.ny;
  const int hc = sx.half - ngb + 1, nc = sx.node - ngb;   // Ex/Bz and Ey column bases
  const int nr = sy.node - ngb, hr = sy.half - ngb + 1;   // Ex and Ey/Bz row bases
  // tap (i, j) of each component
  auto ex = [&](int i, int j) -> float {
    if constexpr (WIN) return sEx[(hc + i - w.sx0) + (nr + j - w.sy0) * w.sstr];
    if (CHECKED && !in_box(hc + i, nr + j, nx + 2, ny + 1)) return 0.0f;
    return __ldg(f.Ex + (hc + i) + (nr + j) * (nx + 2));
  };
  auto ey = [&](int i, int j) -> float {
    if constexpr (WIN) return sEy[(nc + i - w.sx0) + (hr + j - w.sy0) * w.sstr];
    if (CHECKED && !in_box(nc + i, hr + j, nx + 1, ny + 2)) return 0.0f;
    return __ldg(f.Ey + (nc + i) + (hr + j) * (nx + 1));
  };
  auto bz = [&](int i, int j) -> float {
    if constexpr (WIN) return sBz[(hc + i - w.sx0) + (hr + j - w.sy0) * w.sstr];
    if (CHECKED && !in_box(hc + i, hr + j, nx + 2, ny + 2)) return 0.0f;
    return __ldg(f.Bz + (hc + i) + (hr + j) * (nx + 2));
  };
#pragma unroll
  for (int j = 0; j <= ORDER; ++j) {
    float rx = 0.0f, ry = 0.0f, rz = 0.0f;
#pragma unroll
    for (int i = 0; i <= ORDER; ++i) {
      rx += wxh[i] * ex(i, j);
      ry += wxn[i] * ey(i, j);
      if constexpr (!BZU) rz += wxh[i] * bz(i, j);
    }
    Epx += wyn[j] * rx;
    Epy += wyh[j] * ry;
    if constexpr (!BZU) Bpz += wyh[j] * rz;
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

// Boris rotation factors for a magnetic field Bz (src/Particle.mm:157-209),
// every operation explicitly rounded: fe scales the half-step electric kick
// (constE * fN1), btz is the rotation parameter t (times fN1 for the order-4/6
// corrections) and ssz = 2 t / (1 + t0^2). Uniform Bz makes them constants of
// the launch, computed once per thread instead of once per particle.
struct BorisFactors {
  float fe, btz, ssz;
};
__device__ __forceinline__ BorisFactors boris_factors(float Bz, float constE, float constB, int boris_order) {
  const float t0 = __fmul_rn(constB, Bz);
  const float tt = __fmul_rn(t0, t0);
  float fN1 = 1.0f;
  if (boris_order == 4)
    fN1 = __fadd_rn(1.0f, __fdiv_rn(tt, 3.0f));
  else if (boris_order == 6)
    fN1 = __fadd_rn(__fadd_rn(1.0f, __fdiv_rn(tt, 3.0f)), __fdiv_rn(__fmul_rn(__fmul_rn(2.0f, tt), tt), 15.0f));
  BorisFactors b;
  b.fe = __fmul_rn(constE, fN1);
  b.btz = __fmul_rn(t0, fN1);
  b.ssz = __fdiv_rn(__fmul_rn(2.0f, b.btz), __fadd_rn(1.0f, tt));
  return b;
}

// Periodic wrap of a cell index into [ngb, ngb + n): one conditional add or
// subtract for a move of less than a period, the remainder otherwise.
__device__ __forceinline__ int wrap_periodic(int i, int ngb, int n) {
  int d = i - ngb;
  if (d < 0)
    d += n;
  else if (d >= n)
    d -= n;
  if (d < 0 || d >= n) d = ((d % n) + n) % n;
  return ngb + d;
}

__device__ __forceinline__ bool interior(const GridDims& g, int ix, int iy) {
  return ix >= g.ngb && ix < g.ngb + g.ngx && iy >= g.ngb && iy < g.ngb + g.ngy;
}

template <int ORDER, bool PUSH, bool DEP, bool DET, bool CUR, bool BZU>
__host__ __device__ constexpr size_t smem_bytes() {
  return (PUSH ? (BZU ? 2 : 3) * size_t(kWin) * sizeof(float) : 0) +
         (DEP ? DepositLayout<ORDER, CUR, DET>::kBytes : 0);
}

// Phases A and B of a chunk (shared by the push / deposit kernels): the box
// of the chunk's cells, the shared-memory field window or gather table
// covering it, and the cleared deposit window. Returns the window (also in s_w).
// TMA: the Ex / Ey tiles are staged by bulk tensor copies from the pitched
// copies (tm, when valid; bar: the CTA's initialised mbarrier), which fill
// elements outside the arrays with zero as the per-thread loads do; a copy
// that does not complete within the wait's bound makes the threads load the
// tiles per thread instead (same values); staged chunks are
// counted in cnt->n_tma, time-outs in cnt->err.
template <int ORDER, bool PUSH, bool DEP, bool DET, bool CUR, bool BZU, bool TMA = false, int PER = kPer>
__device__ __forceinline__ Window chunk_setup(const GridDims& g, const ParticleArrays& p, const FieldPtrs& f,
                                            uint32_t n, uint32_t base, int tid, int lane, int wid, float* sEx,
                                            float* sEy, float* sBz, int* sDep, int (*s_red)[kThreads / 32],
                                            Window& s_w, int32_t& s_ref, const FieldMaps* tm = nullptr,
                                            uint32_t bar = 0, SpeciesCounters* cnt = nullptr, bool tables = true) {
  using DL = DepositLayout<ORDER, CUR, DET>;
  constexpr bool kTab = PUSH && BZU && ORDER == 3 && !DET && !CUR;
  const int ngb = g.ngb;
  // ---- phase A: box of the chunk's cells (re-read from L1 below). Only
  // particles within kReach cells of the chunk's middle particle count, so
  // that a few strays (holes filled by compaction, injected particles) do not
  // blow up the box; particles outside it use the global paths.
  // (a thread's cells are loaded before the barrier that publishes the
  // middle particle, so the two loads overlap)
  int32_t cls[PER];
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    const uint32_t k = base + uint32_t(i * kThreads + tid);
    cls[i] = k < n ? p.cell[k] : -1;
  }
  if (tid == 0) {
    const uint32_t rest = n - base;
    constexpr uint32_t chunk = uint32_t(kThreads * PER);
    const int32_t rc = p.cell[base + (rest < chunk ? rest / 2 : chunk / 2)];
    s_ref = (rc >= 0 && interior(g, cell_ix(rc), cell_iy(rc))) ? rc : -1;
  }
  __syncthreads();
  const int32_t ref = s_ref;
  const int rx = ref >= 0 ? cell_ix(ref) : 0, ry = ref >= 0 ? cell_iy(ref) : 0;
  const int reach = ref >= 0 ? kReach : INT_MAX / 2;
  int mnx = INT_MAX, mny = INT_MAX, mxx = INT_MIN, mxy = INT_MIN;
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    const int32_t cl = cls[i];
    if (cl >= 0) {
      const int ix = cell_ix(cl), iy = cell_iy(cl);
      if (interior(g, ix, iy) && abs(ix - rx) <= reach && abs(iy - ry) <= reach) {
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
    w.priv = 0;
    w.ps = 1;
    w.tab = 0;
    w.tbw = w.tbh = 1;
    w.xrs = w.yrs = w.yoff = 0;
    w.tma = w.sbox = w.soff = 0;
    w.sx0 = w.sy0 = 0;
    w.sstr = w.shh = 1;
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
      w.ds = w.dw + (((ORDER + 1 - w.dw) % 32) + 32) % 32;
      w.use = (w.ds * w.dh <= kWin && w.gw * w.gh <= kWin) ? 1 : 0;
      w.priv = 0;
      w.ps = (kPW * w.dh) | 1;
      if (DEP && DL::kSingle && w.use && w.dw <= kPW && 32 * w.ps + 3 <= kPrivWords) w.priv = 1;
      w.tbw = w.mxx - w.mnx + 1;
      w.tbh = w.mxy - w.mny + 1;
      w.xrs = tab_row_stride(w.tbw + 1);
      w.yrs = tab_row_stride(w.tbw);
      w.yoff = w.tbh * w.xrs;
      w.tab = (kTab && tables && w.use && w.yoff + (w.tbh + 1) * w.yrs <= kTabFloat4) ? 1 : 0;
      w.sx0 = w.gx0;
      w.sy0 = w.gy0;
      w.sstr = w.gw;
      w.shh = w.gh;
      if constexpr (TMA && PUSH) {
        // gx0 = mnx - ngb >= 0 (box cells are interior); the copy starts at
        // the multiple of 4 columns at or below it
        const int x0 = w.gx0 & ~3, y0 = w.gy0;
        if (w.use && tm->valid && (smem_u32(sEx) & 127u) == 0) {
          if (w.tab) {
            // taps read by the table build: Ex columns gx0 .. gx0 + tbw + 3,
            // rows gy0 .. gy0 + tbh + 2; Ey columns gx0 .. gx0 + tbw + 2,
            // rows gy0 .. gy0 + tbh + 3; both tiles after the tables
            const int b = field_box(w.gx0 - x0 + w.tbw + 4, w.tbh + 4);
            const int off = ((w.yoff + (w.tbh + 1) * w.yrs) * 16 + 127) & ~127;
            if (b >= 0 && off + 8 * field_box_w(b) * field_box_h(b) <= 2 * kWin * int(sizeof(float))) {
              w.tma = 1;
              w.sbox = b;
              w.soff = off;
            }
          } else {
            const int b = field_box(w.gx0 - x0 + w.gw, w.gh);
            if (b >= 0) {
              w.tma = 1;
              w.sbox = b;
            }
          }
          if (w.tma) {
            w.sx0 = x0;
            w.sstr = field_box_w(w.sbox);
            w.shh = field_box_h(w.sbox);
            const uint32_t fb = 4u * uint32_t(w.sstr * w.shh);  // bytes per tile, a multiple of 128
            const uint32_t dx = smem_u32(sEx) + uint32_t(w.soff);
            const uint32_t dy = w.tab ? dx + fb : smem_u32(sEy);
            mbar_expect_tx(bar, 2 * fb);
            tma_tile(dx, &tm->ex[w.sbox], x0, y0, bar);
            tma_tile(dy, &tm->ey[w.sbox], x0, y0, bar);
          }
        }
      }
    }
    s_w = w;
  }
  __syncthreads();
  const Window w = s_w;
  // clear the deposit window while the field copies are in flight (it does
  // not overlap their destination)
  if constexpr (DEP) {
    if (w.use) {
      if (w.priv) {
        int4* z = reinterpret_cast<int4*>(sDep);  // 32 * ps rounded up to 4 words stays within kPrivWords
        for (int e = tid; e < (32 * w.ps + 3) / 4; e += kThreads) z[e] = make_int4(0, 0, 0, 0);
      } else {
        const int used = w.ds * w.dh;
        for (int e = tid; e < DL::kArrays * DL::kCopies * used; e += kThreads)
          sDep[(e / used) * DL::kStride + e % used] = 0;
      }
    }
  }
  bool staged = false;  // the bulk copies have landed
  if constexpr (TMA && PUSH) {
    if (w.tma) {
      staged = mbar_wait0(bar);
      if (!staged) atomicAdd(&cnt->err, 1u);
      if (tid == 0) atomicAdd(&cnt->n_tma, 1u);
    }
    if (tid == 0 && w.tab) atomicAdd(&cnt->n_tab, 1u);
    if (tid == 0 && w.priv) atomicAdd(&cnt->n_priv, 1u);
  }

  // ---- phase B: stage the field window (the deposit window was cleared above)
  if (w.use) {
    if (kTab && w.tab) {
      // four polynomials per box cell: Ex below / above the half offset, Ey likewise
      const int nx = g.nx;
      // Ex: one polynomial per half-shifted column h (half = mnx - 1 + h, h in
      // [0, tbw]) and row; Ey: per column and half-shifted row (as h in y).
      float4* tb = reinterpret_cast<float4*>(sEx);
      const int nxe = (w.tbw + 1) * w.tbh, total = nxe + w.tbw * (w.tbh + 1);
      for (int e = tid; e < total; e += kThreads) {
        const bool ex = e < nxe;
        const int t = ex ? e : e - nxe;
        const int rw = ex ? w.tbw + 1 : w.tbw;  // entries per table row
        const int col = t % rw, row = t / rw;
        const int c0 = w.mnx - ngb + col, r0 = w.mny - ngb + row;  // taps c0..c0+3, r0..r0+3
        float F[16];
        if (staged) {
          const float* src = reinterpret_cast<const float*>(reinterpret_cast<const unsigned char*>(sEx) + w.soff) +
                             (ex ? 0 : w.sstr * w.shh) + (c0 - w.sx0) + (r0 - w.sy0) * w.sstr;
#pragma unroll
          for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int i = 0; i < 4; ++i) F[i + 4 * j] = src[i + j * w.sstr];
        } else {
          const float* src = ex ? f.Ex : f.Ey;
          const int stride = ex ? nx + 2 : nx + 1;
#pragma unroll
          for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int i = 0; i < 4; ++i) F[i + 4 * j] = __ldg(src + (c0 + i) + (r0 + j) * stride);
        }
        tab_build(F, tb + (ex ? row * w.xrs : w.yoff + row * w.yrs) + kTabEntry * col);
      }
    } else if constexpr (PUSH) {
      const int nx = g.nx, ny = g.ny;
      for (int e = tid; !staged && e < w.sstr * w.shh; e += kThreads) {
        const int col = w.sx0 + e % w.sstr, row = w.sy0 + e / w.sstr;
        sEx[e] = in_box(col, row, nx + 2, ny + 1) ? __ldg(f.Ex + col + row * (nx + 2)) : 0.0f;
        sEy[e] = in_box(col, row, nx + 1, ny + 2) ? __ldg(f.Ey + col + row * (nx + 1)) : 0.0f;
        if constexpr (!BZU) sBz[e] = in_box(col, row, nx + 2, ny + 2) ? __ldg(f.Bz + col + row * (nx + 2)) : 0.0f;
      }
    }
  }
  __syncthreads();

  return w;
}

// Phase D: flush the chunk's deposit window with one global atomic per node.
template <int ORDER, bool DET, bool CUR>
__device__ __forceinline__ void chunk_flush(const GridDims& g, const PushConsts& c, const DepositTargets& d,
                                            const int* sDep, const Window& w, int tid) {
  using DL = DepositLayout<ORDER, CUR, DET>;
  if (DL::kSingle && w.priv) {
    const int nx = g.nx, ny = g.ny;
    const double fr = double(c.scale) / double(1 << DL::kQBits);
    for (int e = tid; e < kPW * w.dh; e += kThreads) {
      const int cc = e % kPW;
      if (cc >= w.dw) continue;
      const int col = w.dx0 + cc, row = w.dy0 + e / kPW;
      // each copy word stays below 2^31 (DepositLayout); the 32 together
      // fit 32 unsigned bits for orders 3 and 5, not for order 1 (weights up
      // to 1), which sums in 64 bits
      using Sum = std::conditional_t<DL::kPrivSum32, uint32_t, unsigned long long>;
      Sum r = 0;
#pragma unroll 8
      for (int q = 0; q < 32; ++q) r += Sum(uint32_t(sDep[q * w.ps + e]));
      if (r != 0 && in_box(col, row, nx + 1, ny + 1)) atomicAdd(d.f64_rho + col + row * (nx + 1), double(r) * fr);
    }
  } else if (w.use) {
    const int nx = g.nx, ny = g.ny;
    for (int e = tid; e < w.ds * w.dh; e += kThreads) {
      if (e % w.ds >= w.dw) continue;  // stride padding, never written
      const int col = w.dx0 + e % w.ds, row = w.dy0 + e / w.ds;
      long long r = 0, a = 0, b = 0;
#pragma unroll
      for (int q = 0; q < DL::kCopies; ++q) {
        if constexpr (DL::kSingle)
          r += static_cast<long long>(sDep[q * DL::kStride + e]);
        else
          r += wsum(sDep, (0 * DL::kCopies + q) * DL::kStride + e, (1 * DL::kCopies + q) * DL::kStride + e);
        if constexpr (CUR) {
          a += wsum(sDep, (2 * DL::kCopies + q) * DL::kStride + e, (3 * DL::kCopies + q) * DL::kStride + e);
          b += wsum(sDep, (4 * DL::kCopies + q) * DL::kStride + e, (5 * DL::kCopies + q) * DL::kStride + e);
        }
      }
      // fast mode: FP64 sums of w * scale (currents w * scale * v)
      const double unit = DL::kSingle ? 1.0 / double(1 << DL::kQBits) : 0x1p-40;
      const double fr = double(c.scale) * unit, fj = fr * 2.99792458e10;
      if (r != 0 && in_box(col, row, nx + 1, ny + 1)) {
        if constexpr (DET)
          gadd(d.acc_rho + col + row * (nx + 1), r);
        else
          atomicAdd(d.f64_rho + col + row * (nx + 1), double(r) * fr);
      }
      if constexpr (CUR) {
        if (a != 0 && in_box(col, row, nx + 2, ny + 1)) {
          if constexpr (DET)
            gadd(d.acc_jx + col + row * (nx + 2), a);
          else
            atomicAdd(d.f64_jx + col + row * (nx + 2), double(a) * fj);
        }
        if (b != 0 && in_box(col, row, nx + 1, ny + 2)) {
          if constexpr (DET)
            gadd(d.acc_jy + col + row * (nx + 1), b);
          else
            atomicAdd(d.f64_jy + col + row * (nx + 1), double(b) * fj);
        }
      }
    }
  }
}

// Per-warp sums of the push tallies and kinetic energy into the counters.
__device__ __forceinline__ void flush_tallies(uint32_t tally, double ke, const PushConsts& c, SpeciesCounters* cnt,
                                              int lane) {
  auto field = [&](int f) { return warp_sum((tally >> (4 * f)) & 0xFu); };
  const uint32_t s_dead = field(0);
  const uint32_t s_w0 = field(1), s_w1 = field(2);
  const uint32_t s_w2 = field(3), s_w3 = field(4);
  const uint32_t s_inv = field(5), s_slow = field(6);
  const double s_ke = warp_sum(ke) * c.ke_half_m * c.ke_w;  // kinetic energy, src/Particle.mm:980-982
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

template <int ORDER, bool PUSH, bool DEP, bool DET, bool CUR, bool BZU>
__global__ void __launch_bounds__(kThreads, ORDER == 5 ? 2 : (PUSH && (!BZU || !DEP) ? 3 : 4)) k_pic(GridDims g, ParticleArrays p, FieldPtrs f, PushConsts c,
                                                  int boris_order, DepositTargets d, SpeciesCounters* cnt,
                                                  uint32_t* dead_bits, int injected_only) {
  using DL = DepositLayout<ORDER, CUR, DET>;
  // Gather tables (they replace the Ex/Ey windows) round differently from the
  // stencil sum that every other path evaluates, so a particle's field would
  // depend on its chunk's box; the deterministic mode (DET, also passed to its
  // pushes without deposit) keeps the stencil sum everywhere.
  // (not with currents: the two paths together exceed the 64 registers of order 3)
  constexpr bool kTab = PUSH && BZU && ORDER == 3 && !DET && !CUR;
  extern __shared__ __align__(128) unsigned char smem[];
  float* sEx = reinterpret_cast<float*>(smem);
  float* sEy = sEx + (PUSH ? kWin : 0);
  float* sBz = sEy + (PUSH ? kWin : 0);
  // copy c of array a starts at (a * kCopies + c) * kStride; arrays: rho hi,
  // rho lo, jx hi, jx lo, jy hi, jy lo
  int* sDep = reinterpret_cast<int*>(smem + (PUSH ? (BZU ? 2 : 3) * size_t(kWin) * sizeof(float) : 0));
  __shared__ int s_red[4][kThreads / 32];
  __shared__ Window s_w;
  __shared__ int32_t s_ref;

  const uint32_t n = cnt->n;
  const uint32_t first = (!PUSH && injected_only) ? n - cnt->n_injected : 0u;
  const uint32_t base = first + blockIdx.x * uint32_t(kChunk);
  if (base >= n) return;  // uniform over the block
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int ngb = g.ngb;
  const int copy = (lane / DL::kN2) % DL::kCopies;
  WinPtrs sw;
  sw.rho = static_cast<uint32_t>(__cvta_generic_to_shared(sDep + copy * DL::kStride));

  constexpr bool kVel = PUSH || CUR;
  int32_t q_cell = -1;
  float q_ox = 0.0f, q_oy = 0.0f, q_vx = 0.0f, q_vy = 0.0f, q_vz = 0.0f;
  auto fetch = [&](uint32_t k) {
    if (k < n) {
      q_cell = p.cell[k];
      q_ox = p.ox[k];
      q_oy = p.oy[k];
      if constexpr (kVel) {
        q_vx = p.vx[k];
        q_vy = p.vy[k];
      }
      if constexpr (PUSH) q_vz = p.vz[k];
    }
  };
  fetch(base + uint32_t(tid));  // in flight during the chunk set-up
  const Window w = chunk_setup<ORDER, PUSH, DEP, DET, CUR, BZU>(g, p, f, n, base, tid, lane, wid, sEx, sEy, sBz, sDep,
                                                                s_red, s_w, s_ref);
  const uint32_t priv_base = static_cast<uint32_t>(__cvta_generic_to_shared(sDep)) + 4u * uint32_t(lane * w.ps);

  // ---- phase C: particles. The loads of a thread's next particle are issued
  // before the current one is processed, so that their latency overlaps the
  // arithmetic (the kernel is otherwise bound by the load round trip).
  const BorisFactors bzu = BZU ? boris_factors(c.bz_uniform, c.constE, c.constB, boris_order) : BorisFactors{};
  // per-thread tallies in 4-bit fields of one register (at most kPer each):
  // dead [0,4), wall w [4(w+1), 4(w+2)), invalid [20,24), slow [24,28)
  static_assert(kPer < 16, "tally fields are 4 bits wide");
  uint32_t tally = 0;
  double ke = 0.0;  // sum of |v|^2 (FP64) over this thread's pushed particles
#pragma unroll 1
  for (int i = 0; i < kPer; ++i) {
    const uint32_t k = base + uint32_t(i * kThreads + tid);
    const int32_t cell = q_cell;
    const float l_ox = q_ox, l_oy = q_oy, l_vx = q_vx, l_vy = q_vy, l_vz = q_vz;
    if (i + 1 < kPer) fetch(k + uint32_t(kThreads));
    int fl = 0;
    if (k < n) {
      if (cell < 0) {
        fl = -cell;  // flagged before this push and not yet compacted: keep the flag
      } else {
        int ix = cell_ix(cell), iy = cell_iy(cell);
        float ox = l_ox, oy = l_oy;
        const bool inside = interior(g, ix, iy);
        const bool in_box_win = w.use && ix >= w.mnx && ix <= w.mxx && iy >= w.mny && iy <= w.mxy;
        if constexpr (!PUSH) {
          const Stagger sx = stagger(ix, ox), sy = stagger(iy, oy);
          float wxn[ORDER + 1], wxh[ORDER + 1], wyn[ORDER + 1], wyh[ORDER + 1];
          shape<ORDER>(sx.hnode, wxn);
          shape<ORDER>(sy.hnode, wyn);
          float vx = 0.0f, vy = 0.0f;
          if constexpr (CUR) {
            shape<ORDER>(sx.hhalf, wxh);
            shape<ORDER>(sy.hhalf, wyh);
            vx = l_vx;
            vy = l_vy;
          }
          if (DL::kSingle && in_box_win && w.priv)
            deposit_priv<ORDER>(w, priv_base, ngb, sx, sy, wxn, wyn);
          else if (in_box_win && sublight<CUR>(vx, vy))
            deposit_one<ORDER, DET, CUR, true, false>(g, w, lane, sx, sy, wxn, wxh, wyn, wyh, c.scale, vx, vy, d, sw);
          else if (inside)
            deposit_one<ORDER, DET, CUR, false, false>(g, w, lane, sx, sy, wxn, wxh, wyn, wyh, c.scale, vx, vy, d, sw);
          else
            deposit_one<ORDER, DET, CUR, false, true>(g, w, lane, sx, sy, wxn, wxh, wyn, wyh, c.scale, vx, vy, d, sw);
        } else {
          float vx = l_vx, vy = l_vy, vz = l_vz;
          const Stagger sx = stagger(ix, ox), sy = stagger(iy, oy);
          float wxn[ORDER + 1], wxh[ORDER + 1], wyn[ORDER + 1], wyh[ORDER + 1];
          float Epx = 0.0f, Epy = 0.0f, Bpz = 0.0f;
          if (kTab && in_box_win && s_w.tab) {  // read from shared memory: no register held across the loop
            const float4* tb = reinterpret_cast<const float4*>(sEx);
            const int cx = ix - w.mnx, cy = iy - w.mny;
            Epx = tab_eval(tb + cy * s_w.xrs + kTabEntry * (cx + (ox >= 0.5f ? 1 : 0)), sx.hhalf, oy);
            Epy = tab_eval(tb + s_w.yoff + (cy + (oy >= 0.5f ? 1 : 0)) * s_w.yrs + kTabEntry * cx, ox, sy.hhalf);
          } else {
            shape<ORDER>(sx.hnode, wxn);
            shape<ORDER>(sx.hhalf, wxh);
            shape<ORDER>(sy.hnode, wyn);
            shape<ORDER>(sy.hhalf, wyh);
            if (in_box_win)
              gather<ORDER, BZU, true, false>(g, f, w, sx, sy, wxn, wxh, wyn, wyh, sEx, sEy, sBz, Epx, Epy, Bpz);
            else if (inside)
              gather<ORDER, BZU, false, false>(g, f, w, sx, sy, wxn, wxh, wyn, wyh, sEx, sEy, sBz, Epx, Epy, Bpz);
            else
              gather<ORDER, BZU, false, true>(g, f, w, sx, sy, wxn, wxh, wyn, wyh, sEx, sEy, sBz, Epx, Epy, Bpz);
          }
          if (!in_box_win) tally += 1u << 24;
          // Boris push (src/Particle.mm:157-209); Ez, Bx, By are identically
          // zero in the reference's gather (:134-139).
          const BorisFactors bf = BZU ? bzu : boris_factors(Bpz, c.constE, c.constB, boris_order);
          const float btz = bf.btz, ssz = bf.ssz;
          const float etx = __fmul_rn(bf.fe, Epx), ety = __fmul_rn(bf.fe, Epy);
          const float umx = vx + etx, umy = vy + ety, umz = vz;
          const float v0x = umx + umy * btz;
          const float v0y = umy - umx * btz;
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
          } else if (!interior(g, ix, iy)) {  // boundary conditions act only on a particle that left the grid
            if (c.bc[0] == 0) ix = wrap_periodic(ix, ngb, g.ngx);
            if (c.bc[2] == 0) iy = wrap_periodic(iy, ngb, g.ngy);
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
            const float vv = __fadd_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)), __fmul_rn(vz, vz));
            ke += double(vv);
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
              if (DL::kSingle && in_win && w.priv)
                deposit_priv<ORDER>(w, priv_base, ngb, nsx, nsy, wxn, wyn);
              else if (in_win && sublight<CUR>(vx, vy))
                deposit_one<ORDER, DET, CUR, true, false>(g, w, lane, nsx, nsy, wxn, wxh, wyn, wyh, c.scale, vx, vy, d,
                                                          sw);
              else
                deposit_one<ORDER, DET, CUR, false, false>(g, w, lane, nsx, nsy, wxn, wxh, wyn, wyh, c.scale, vx, vy, d,
                                                           sw);
            }
          } else {
            p.cell[k] = -fl;
          }
        }
      }
      if (fl)  // includes particles flagged before this push and not yet compacted
        tally += 1u + (fl <= 4 ? 1u << (4 * fl) : 1u << 20);
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
    chunk_flush<ORDER, DET, CUR>(g, c, d, sDep, w, tid);
  }
  if constexpr (PUSH) flush_tallies(tally, ke, c, cnt, lane);
}

// Node-centred weights of a particle at offsets h = (hx, hy) for both axes at
// once: shape<ORDER> evaluated on packed FP32 pairs (each half rounds exactly
// like the scalar intrinsics), with the x weights scaled by sx, a power of
// two folded into the constants (scaling by 2^q commutes with every rounding
// step, so wx[t] == sx * shape<ORDER>(hx)[t] and wy[t] == shape<ORDER>(hy)[t]
// bit for bit).
template <int ORDER>
__device__ __forceinline__ void shape2(float2 h, float sx, float (&wx)[ORDER + 1], float (&wy)[ORDER + 1]) {
  auto cp = [sx](float v) { return make_float2(v * sx, v); };
  auto c1 = [](float v) { return make_float2(v, v); };
  if constexpr (ORDER == 1) {
    const float2 u = __ffma2_rn(h, cp(-1.0f), cp(1.0f));  // sx (1 - h), 1 - h
    const float2 v = __fmul2_rn(h, cp(1.0f));
    wx[0] = u.x, wy[0] = u.y, wx[1] = v.x, wy[1] = v.y;
  } else if constexpr (ORDER == 3) {
    constexpr float c6 = 1.0f / 6.0f, c23 = 2.0f / 3.0f;
    const float2 u = __ffma2_rn(h, c1(-1.0f), c1(1.0f));
    const float2 h2 = __fmul2_rn(h, h), u2 = __fmul2_rn(u, u);
    const float2 w0 = __fmul2_rn(__fmul2_rn(u2, u), cp(c6));
    const float2 w1 = __ffma2_rn(h2, __ffma2_rn(h, cp(0.5f), cp(-1.0f)), cp(c23));
    const float2 w2 = __ffma2_rn(u2, __ffma2_rn(u, cp(0.5f), cp(-1.0f)), cp(c23));
    const float2 w3 = __fmul2_rn(__fmul2_rn(h2, h), cp(c6));
    wx[0] = w0.x, wy[0] = w0.y, wx[1] = w1.x, wy[1] = w1.y;
    wx[2] = w2.x, wy[2] = w2.y, wx[3] = w3.x, wy[3] = w3.y;
  } else {
    constexpr float c120 = 1.0f / 120.0f;
    constexpr float a0 = 26.0f / 120.0f, a1 = -50.0f / 120.0f, a2 = 20.0f / 120.0f, a3 = 20.0f / 120.0f,
                    a4 = -20.0f / 120.0f, a5 = 5.0f / 120.0f;
    constexpr float b0 = 11.0f / 20.0f, b2 = -0.5f, b4 = 0.25f, b5 = -1.0f / 12.0f;
    const float2 u = __ffma2_rn(h, c1(-1.0f), c1(1.0f));
    const float2 h2 = __fmul2_rn(h, h), u2 = __fmul2_rn(u, u);
    const float2 w0 = __fmul2_rn(__fmul2_rn(__fmul2_rn(u2, u2), u), cp(c120));
    const float2 w5 = __fmul2_rn(__fmul2_rn(__fmul2_rn(h2, h2), h), cp(c120));
    const float2 w1 = __ffma2_rn(
        h, __ffma2_rn(h, __ffma2_rn(h, __ffma2_rn(h, __ffma2_rn(h, cp(a5), cp(a4)), cp(a3)), cp(a2)), cp(a1)), cp(a0));
    const float2 w4 = __ffma2_rn(
        u, __ffma2_rn(u, __ffma2_rn(u, __ffma2_rn(u, __ffma2_rn(u, cp(a5), cp(a4)), cp(a3)), cp(a2)), cp(a1)), cp(a0));
    const float2 w2 = __ffma2_rn(h2, __ffma2_rn(h2, __ffma2_rn(h, cp(b5), cp(b4)), cp(b2)), cp(b0));
    const float2 w3 = __ffma2_rn(u2, __ffma2_rn(u2, __ffma2_rn(u, cp(b5), cp(b4)), cp(b2)), cp(b0));
    wx[0] = w0.x, wy[0] = w0.y, wx[1] = w1.x, wy[1] = w1.y, wx[2] = w2.x, wy[2] = w2.y;
    wx[3] = w3.x, wy[3] = w3.y, wx[4] = w4.x, wy[4] = w4.y, wx[5] = w5.x, wy[5] = w5.y;
  }
}

// Push + fused deposit for the atomic mode without currents in a uniform Bz
// (the 512 x 512 benchmark workload and most ensemble members). Phases A, B
// and D are k_pic's; phase C evaluates the same expressions in the same order
// (gather tables for order 3, staged windows for orders 1 and 5, Boris,
// move, boundary conditions, lane-private or rotated single-word deposit
// windows), so particle states and window sums are bit-identical to
// k_pic<ORDER, 1, 1, 0, 0, 1>. What differs is the bookkeeping around them:
// the window parameters a particle needs stay in registers with the box
// origin folded into the shared-memory base addresses (one multiply-add per
// address), box tests are one unsigned comparison per axis, and the
// per-particle reads of the window descriptor from shared memory are gone.
template <int ORDER, int PER>
__global__ void __launch_bounds__(kThreads, ORDER == 5 ? 2 : 4)
    k_push_fast(GridDims g, ParticleArrays p, FieldPtrs f, PushConsts c, int boris_order, DepositTargets d,
                SpeciesCounters* cnt, uint32_t* dead_bits, const __grid_constant__ FieldMaps tm) {
  using DL = DepositLayout<ORDER, false, false>;
  constexpr int N = ORDER + 1;
  constexpr bool kTab = ORDER == 3;
  extern __shared__ __align__(128) unsigned char smem[];
  float* sEx = reinterpret_cast<float*>(smem);
  float* sEy = sEx + kWin;
  int* sDep = reinterpret_cast<int*>(smem + 2 * size_t(kWin) * sizeof(float));
  __shared__ int s_red[4][kThreads / 32];
  __shared__ Window s_w;
  __shared__ int32_t s_ref;
  __shared__ __align__(8) uint64_t s_bar;  // field staging (one use)

  const uint32_t n = cnt->n;
  const uint32_t base = blockIdx.x * uint32_t(kThreads * PER);
  if (base >= n) return;  // uniform over the block
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int ngb = g.ngb;
  const uint32_t bar = smem_u32(&s_bar);
  int32_t q_cell = -1;
  float q_ox = 0.0f, q_oy = 0.0f, q_vx = 0.0f, q_vy = 0.0f, q_vz = 0.0f;
  auto fetch = [&](uint32_t k) {
    if (k < n) {
      q_cell = p.cell[k];
      q_ox = p.ox[k];
      q_oy = p.oy[k];
      q_vx = p.vx[k];
      q_vy = p.vy[k];
      q_vz = p.vz[k];
    }
  };
  fetch(base + uint32_t(tid));  // in flight during the chunk set-up
  if (tid == 0) mbar_init1(bar);  // ordered before the copies by phase A's barriers
  const Window w = chunk_setup<ORDER, true, true, false, false, true, true, PER>(
      g, p, f, n, base, tid, lane, wid, sEx, sEy, nullptr, sDep, s_red, s_w, s_ref, &tm, bar, cnt, c.no_tables == 0);
  WinPtrs sw;
  sw.rho = static_cast<uint32_t>(__cvta_generic_to_shared(sDep + ((lane / DL::kN2) % DL::kCopies) * DL::kStride));

  // ---- phase C
  const BorisFactors bz = boris_factors(c.bz_uniform, c.constE, c.constB, boris_order);
  const bool use = w.use != 0;
  const bool tab = kTab && use && w.tab;
  const bool priv = use && w.priv;
  const int mnx = w.mnx, mny = w.mny;
  const uint32_t bw = uint32_t(w.mxx - w.mnx), bh = uint32_t(w.mxy - w.mny);
  // deposit window in cells: [mnx - kMargin, mxx + kMargin] x [mny - kMargin, mxy + kMargin]
  const int wx0 = mnx - kMargin, wy0 = mny - kMargin;
  const uint32_t ww = bw + 2 * kMargin, wh = bh + 2 * kMargin;
  // gather table (float4 units): Ex entry of box cell (cx, cy) and upper half
  // ux at cy * xrs + 5 (cx + ux), Ey entry at yoff + (cy + uy) * yrs + 5 cx
  const float4* tbx = reinterpret_cast<const float4*>(sEx) - (mny * w.xrs + kTabEntry * mnx);
  const float4* tby = reinterpret_cast<const float4*>(sEx) + w.yoff - (mny * w.yrs + kTabEntry * mnx);
  const int xrs = w.xrs, yrs = w.yrs;
  // lane-private deposit window: node (col, row) of this lane's copy at
  // pbase + 4 (col + row kPW) with col = ix (x node index of the stencil base)
  const uint32_t pbase = static_cast<uint32_t>(__cvta_generic_to_shared(sDep)) + 4u * uint32_t(lane * w.ps) -
                         4u * uint32_t((ngb + w.dx0) + (ngb + w.dy0) * kPW);

  uint32_t tally = 0;
  float ke = 0.0f;  // sum of |v|^2 over this thread's pushed particles (at most PER)
#pragma unroll 1
  for (int i = 0; i < PER; ++i) {
    const uint32_t k = base + uint32_t(i * kThreads + tid);
    const int32_t cell = q_cell;
    float ox = q_ox, oy = q_oy, vx = q_vx, vy = q_vy, vz = q_vz;
    if (i + 1 < PER) fetch(k + uint32_t(kThreads));
    int fl = 0;
    // The gather of a particle in the chunk's box: per-cell polynomial
    // tables (order 3) or the staged windows (which add into Epx, Epy: the
    // caller starts them at zero).
    auto gather_box = [&](int ix, int iy, float ox, float oy, float& Epx, float& Epy) {
      if (tab) {
        const int ux = ox >= 0.5f ? 1 : 0, uy = oy >= 0.5f ? 1 : 0;
        const float hx = ux ? __fsub_rn(ox, 0.5f) : __fadd_rn(ox, 0.5f);
        const float hy = uy ? __fsub_rn(oy, 0.5f) : __fadd_rn(oy, 0.5f);
        Epx = tab_eval(tbx + iy * xrs + kTabEntry * (ix + ux), hx, oy);
        Epy = tab_eval(tby + (iy + uy) * yrs + kTabEntry * ix, ox, hy);
      } else {
        const Stagger sx = stagger(ix, ox), sy = stagger(iy, oy);
        float wxn[N], wxh[N], wyn[N], wyh[N];
        shape<ORDER>(sx.hnode, wxn);
        shape<ORDER>(sx.hhalf, wxh);
        shape<ORDER>(sy.hnode, wyn);
        shape<ORDER>(sy.hhalf, wyh);
        float Bpz = 0.0f;
        gather<ORDER, true, true, false>(g, f, w, sx, sy, wxn, wxh, wyn, wyh, sEx, sEy, nullptr, Epx, Epy, Bpz);
      }
    };
    // Boris push (src/Particle.mm:157-209) with the launch's Bz factors
    auto boris = [&](float Epx, float Epy, float& vx, float& vy, float& vz) {
      const float etx = __fmul_rn(bz.fe, Epx), ety = __fmul_rn(bz.fe, Epy);
      const float umx = vx + etx, umy = vy + ety, umz = vz;
      const float v0x = umx + umy * bz.btz;
      const float v0y = umy - umx * bz.btz;
      const float upx = umx + v0y * bz.ssz;
      const float upy = umy - v0x * bz.ssz;
      vx = upx + c.constE * Epx;
      vy = upy + c.constE * Epy;
      vz = umz;
    };
    // Store, kinetic energy and deposit of a particle that is live, interior
    // and inside the deposit window after the move.
    auto store_deposit_win = [&](int ix, int iy, float ox, float oy, float vx, float vy, float vz) {
      p.vx[k] = vx;
      p.vy[k] = vy;
      p.vz[k] = vz;
      p.cell[k] = pack_cell(ix, iy);
      p.ox[k] = ox;
      p.oy[k] = oy;
      ke += __fadd_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)), __fmul_rn(vz, vz));
      if (priv) {
        float rx[N], ry[N];  // x weights pre-scaled by the window's fixed-point unit
        shape2<ORDER>(make_float2(ox, oy), float(1 << DL::kQBits), rx, ry);
        priv_add<N>(pbase + 4u * uint32_t(ix + iy * kPW), rx, ry);
      } else {
        float wxn[N], wyn[N], unused[N];
        shape2<ORDER>(make_float2(ox, oy), 1.0f, wxn, wyn);
        deposit_one<ORDER, false, false, true, false>(g, w, lane, stagger(ix, ox), stagger(iy, oy), wxn, unused, wyn,
                                                      unused, c.scale, vx, vy, d, sw);
      }
    };
    // Boundary conditions, store and deposit of any moved particle
    // (src/Particle.mm:212-269); returns the flag.
    auto finish = [&](int ix, int iy, float ox, float oy, float vx, float vy, float vz, bool okx, bool oky) {
      int f = 0;
      if (!(okx && oky) || !isfinite(vz)) {
        f = 5;
      } else if (!interior(g, ix, iy)) {
        if (c.bc[0] == 0) ix = wrap_periodic(ix, ngb, g.ngx);
        if (c.bc[2] == 0) iy = wrap_periodic(iy, ngb, g.ngy);
        if (c.bc[0] == 1 && ix < ngb) f = 1;
        if (c.bc[1] == 1 && ix >= ngb + g.ngx) f = 2;
        if (c.bc[2] == 1 && iy < ngb) f = 3;
        if (c.bc[3] == 1 && iy >= ngb + g.ngy) f = 4;
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
        if (f == 0 && !interior(g, ix, iy)) f = 5;
      }
      if (f != 0) {
        p.vx[k] = vx;
        p.vy[k] = vy;
        p.vz[k] = vz;
        p.cell[k] = -f;
        return f;
      }
      const bool in_win = use && uint32_t(ix - wx0) <= ww && uint32_t(iy - wy0) <= wh;
      if (in_win) {
        store_deposit_win(ix, iy, ox, oy, vx, vy, vz);
      } else {
        p.vx[k] = vx;
        p.vy[k] = vy;
        p.vz[k] = vz;
        p.cell[k] = pack_cell(ix, iy);
        p.ox[k] = ox;
        p.oy[k] = oy;
        ke += __fadd_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)), __fmul_rn(vz, vz));
        float wxn[N], wyn[N], unused[N];
        shape2<ORDER>(make_float2(ox, oy), 1.0f, wxn, wyn);
        deposit_one<ORDER, false, false, false, false>(g, w, lane, stagger(ix, ox), stagger(iy, oy), wxn, unused, wyn,
                                                       unused, c.scale, vx, vy, d, sw);
      }
      return 0;
    };
    int ix = cell_ix(cell), iy = cell_iy(cell);
    const bool inb = use && uint32_t(ix - mnx) <= bw && uint32_t(iy - mny) <= bh;
    // Warps whose 32 particles are all live and inside the staged box take a
    // branch-free path (the usual case for cell-sorted particles); the
    // decisions are warp-uniform, so no lane waits on another's branch.
    if (__all_sync(0xffffffffu, k < n && cell >= 0 && inb)) {
      float Epx = 0.0f, Epy = 0.0f;  // the window gather accumulates into them
      gather_box(ix, iy, ox, oy, Epx, Epy);
      boris(Epx, Epy, vx, vy, vz);
      const bool okx = advance(ix, ox, vx, c.constX);
      const bool oky = advance(iy, oy, vy, c.constY);
      const bool plain = okx && oky && isfinite(vz) && interior(g, ix, iy) && uint32_t(ix - wx0) <= ww &&
                         uint32_t(iy - wy0) <= wh;
      if (__all_sync(0xffffffffu, plain))
        store_deposit_win(ix, iy, ox, oy, vx, vy, vz);
      else
        fl = finish(ix, iy, ox, oy, vx, vy, vz, okx, oky);
    } else if (k < n) {
      if (cell < 0) {
        fl = -cell;  // flagged before this push and not yet compacted: keep the flag
      } else {
        float Epx = 0.0f, Epy = 0.0f;
        if (inb) {
          gather_box(ix, iy, ox, oy, Epx, Epy);
        } else {
          const Stagger sx = stagger(ix, ox), sy = stagger(iy, oy);
          float wxn[N], wxh[N], wyn[N], wyh[N];
          shape<ORDER>(sx.hnode, wxn);
          shape<ORDER>(sx.hhalf, wxh);
          shape<ORDER>(sy.hnode, wyn);
          shape<ORDER>(sy.hhalf, wyh);
          float Bpz = 0.0f;
          if (interior(g, ix, iy))
            gather<ORDER, true, false, false>(g, f, w, sx, sy, wxn, wxh, wyn, wyh, sEx, sEy, nullptr, Epx, Epy, Bpz);
          else
            gather<ORDER, true, false, true>(g, f, w, sx, sy, wxn, wxh, wyn, wyh, sEx, sEy, nullptr, Epx, Epy, Bpz);
          tally += 1u << 24;
        }
        boris(Epx, Epy, vx, vy, vz);
        const bool okx = advance(ix, ox, vx, c.constX);
        const bool oky = advance(iy, oy, vy, c.constY);
        fl = finish(ix, iy, ox, oy, vx, vy, vz, okx, oky);
      }
    }
    if (fl) tally += 1u + (fl <= 4 ? 1u << (4 * fl) : 1u << 20);
    const uint32_t wbase = base + uint32_t(i * kThreads + wid * 32);
    const uint32_t bits = __ballot_sync(0xffffffffu, fl != 0);
    if (lane == 0 && wbase < n) dead_bits[wbase >> 5] = bits;
  }

  // ---- phase D
  __syncthreads();
  chunk_flush<ORDER, false, false>(g, c, d, sDep, w, tid);
  flush_tallies(tally, double(ke), c, cnt, lane);
  // a copy whose wait timed out must not land after the CTA has left
  if (tid == 0 && w.tma) (void)mbar_wait0(bar);
}

template <int ORDER, int PER>
void launch_push_fast(uint32_t nblocks, cudaStream_t s, GridDims g, ParticleArrays p, FieldPtrs f, PushConsts c,
                      int boris, DepositTargets d, SpeciesCounters* cnt, uint32_t* bits, const FieldMaps& tm) {
  auto kern = k_push_fast<ORDER, PER>;
  constexpr size_t bytes = smem_bytes<ORDER, true, true, false, false, true>();
  static std::once_flag once;
  std::call_once(once, [&] { GP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes))); });
  kern<<<nblocks, kThreads, bytes, s>>>(g, p, f, c, boris, d, cnt, bits, tm);
}

template <int ORDER, bool PUSH, bool DEP, bool DET, bool CUR, bool BZU>
void launch_pic(uint32_t nblocks, cudaStream_t s, GridDims g, ParticleArrays p, FieldPtrs f, PushConsts c, int boris,
                DepositTargets d, SpeciesCounters* cnt, uint32_t* bits, int injected_only) {
  auto kern = k_pic<ORDER, PUSH, DEP, DET, CUR, BZU>;
  constexpr size_t bytes = smem_bytes<ORDER, PUSH, DEP, DET, CUR, BZU>();
  static std::once_flag once;  // shared by concurrent runs (ensembles)
  std::call_once(once, [&] { GP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes))); });
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
    if (!dep) {  // DET only selects the bit-reproducible gather here
      if (det)
        bzu ? GP_PIC(false, true, false, true) : GP_PIC(false, true, false, false);
      else
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

}  // namespace

void push(int order, int boris_order, bool dep, bool det, bool cur, bool bzu, GridDims g, ParticleArrays p,
          FieldPtrs f, PushConsts c, DepositTargets d, SpeciesCounters* cnt, uint32_t* dead_bits, uint32_t n_bound,
          cudaStream_t s, const FieldMaps* maps, int chunk_per) {
  // Zero the per-push counters (everything after n).
  GP_CUDA(cudaMemsetAsync(&cnt->n_dead, 0, sizeof(SpeciesCounters) - offsetof(SpeciesCounters, n_dead), s));
  if (n_bound == 0) return;
  const uint32_t nblocks = (n_bound + kChunk - 1) / kChunk;
  if (dep && !det && !cur && bzu) {  // the lean kernel of the common configuration
    static const FieldMaps none{};     // valid = 0: per-thread staging
    const FieldMaps& tm = maps ? *maps : none;
    if (chunk_per != kPer && chunk_per != kPer / 2) throw std::invalid_argument("chunk_per must be 8 or 4");
    const bool half = chunk_per == kPer / 2;
    const uint32_t nb = half ? (n_bound + kChunk / 2 - 1) / (kChunk / 2) : nblocks;
#define GP_FAST(O) \
  half ? launch_push_fast<O, kPer / 2>(nb, s, g, p, f, c, boris_order, d, cnt, dead_bits, tm) \
       : launch_push_fast<O, kPer>(nb, s, g, p, f, c, boris_order, d, cnt, dead_bits, tm)
    switch (order) {
      case 1: GP_FAST(1); break;
      case 3: GP_FAST(3); break;
      case 5: GP_FAST(5); break;
      default: throw std::invalid_argument("WeightingOrder must be 1, 3 or 5");
    }
#undef GP_FAST
    GP_LAUNCH_CHECK();
    return;
  }
  switch (order) {
    case 1: dispatch_pic<1, true>(dep, det, cur, bzu, nblocks, s, g, p, f, c, boris_order, d, cnt, dead_bits, 0); break;
    case 3: dispatch_pic<3, true>(dep, det, cur, bzu, nblocks, s, g, p, f, c, boris_order, d, cnt, dead_bits, 0); break;
    case 5: dispatch_pic<5, true>(dep, det, cur, bzu, nblocks, s, g, p, f, c, boris_order, d, cnt, dead_bits, 0); break;
    default: throw std::invalid_argument("WeightingOrder must be 1, 3 or 5");
  }
  GP_LAUNCH_CHECK();
}

namespace {
__global__ void k_pitch_fields(const float* __restrict__ Ex, const float* __restrict__ Ey, GridDims g,
                               float* __restrict__ Exp, float* __restrict__ Eyp, int pitch) {
  const int nx = g.nx, ny = g.ny;
  const int nEx = (nx + 2) * (ny + 1), nEy = (nx + 1) * (ny + 2);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nEx + nEy; k += gridDim.x * blockDim.x) {
    if (k < nEx)
      Exp[k % (nx + 2) + (k / (nx + 2)) * pitch] = Ex[k];
    else
      Eyp[(k - nEx) % (nx + 1) + ((k - nEx) / (nx + 1)) * pitch] = Ey[k - nEx];
  }
}
}  // namespace

void pitch_fields(const float* Ex, const float* Ey, GridDims g, float* Exp, float* Eyp, cudaStream_t s) {
  const int n = (g.nx + 2) * (g.ny + 1) + (g.nx + 1) * (g.ny + 2);
  k_pitch_fields<<<std::min((n + 255) / 256, 1184), 256, 0, s>>>(Ex, Ey, g, Exp, Eyp, field_pitch(g));
  GP_LAUNCH_CHECK();
}

bool make_field_maps(const float* Exp, const float* Eyp, GridDims g, FieldMaps* maps) {
  *maps = FieldMaps{};
  if ((reinterpret_cast<uintptr_t>(Exp) | reinterpret_cast<uintptr_t>(Eyp)) & 15u) return false;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q{};
  if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !fn) {
    cudaGetLastError();
    return false;
  }
  auto encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  const cuuint64_t stride[1] = {cuuint64_t(field_pitch(g)) * sizeof(float)};  // a multiple of 16 bytes
  const cuuint32_t estr[2] = {1, 1};
  for (int b = 0; b < kFieldBoxes; ++b) {
    const cuuint32_t box[2] = {cuuint32_t(kFieldBoxW[b]), cuuint32_t(kFieldBoxH[b])};
    const cuuint64_t dx[2] = {cuuint64_t(g.nx + 2), cuuint64_t(g.ny + 1)};  // Ex: columns, rows
    const cuuint64_t dy[2] = {cuuint64_t(g.nx + 1), cuuint64_t(g.ny + 2)};  // Ey
    if (encode(&maps->ex[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(Exp), dx, stride, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS ||
        encode(&maps->ey[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(Eyp), dy, stride, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
      *maps = FieldMaps{};
      return false;
    }
  }
  maps->valid = 1;
  return true;
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

}  // namespace kern
}  // namespace gample
