// oracle_core.hpp -- CPU restatement of gample's particle-in-cell step.
//
// TEST INFRASTRUCTURE ONLY. Nothing in the product (gample_b200/, include/)
// may include, link or call this file. Only tests/, __graft_entry__.smoke()
// and bench.py's cpu_baseline leg use it, and only as the checker / the timed
// CPU baseline.
//
// Every function cites the reference file:line it restates (paths are inside
// the gample repository). Arithmetic is templated on the real type R:
//   R = float  -> the reference's own FP32 arithmetic (Metal kernels, float
//                 host buffers), written without FMA contraction
//                 (compile with -ffp-contract=off);
//   R = double -> the FP64 "truth" used to state each GPU result's error.
//
// Parity status: the loader, deposit, ghost folding, Poisson assembly, phi
// reconstruction and gradient are pinned against the reference's own recorded
// timeseries traces (single_darwin_test / uniform_darwin_test CSVs). AMGCL's
// iteration path is not reproducible (library absent); the oracle solves the
// identical CSR system with FP64 CG to the JSON tolerance or tighter.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <string>
#include <tuple>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace oracle {

// ---------------------------------------------------------------- constants
// src/Constant.h:3-25 (CGS-Gaussian)
constexpr double me = 9.10938188e-28;
constexpr double ec = 4.803204197e-10;
constexpr double c_light = 2.99792458e10;
constexpr double kb = 1.3806503e-16;
constexpr double evtoerg = 1.6021764262e-12;
constexpr double ergtoev = 1 / 1.6021764262e-12;
constexpr double eVtoK = 11604;
constexpr double VtosV = 1e8 / c_light;
constexpr double sVtoV = 1 / (1e8 / c_light);
constexpr double JtosJ = 1 / (10 / c_light * 1e4);
constexpr double TtoG = 1e4;
constexpr double PI = 3.141592653589793;  // src/EMField.mm:17, Collision.mm:12

// Boundary-condition codes (strings in the JSON; src/EMField.mm:203-234,
// src/Particle.mm:459-514).
enum FieldBC { FBC_PERIODIC = 0, FBC_DIRICHLET = 1, FBC_NEUMANN = 2, FBC_UNDEF = -1 };
enum ParticleBC { PBC_PERIODIC = 0, PBC_DELETE = 1, PBC_REFLECT = 2 };
enum Wall { XMIN = 0, XMAX = 1, YMIN = 2, YMAX = 3 };

// ------------------------------------------------------------------ RNG
// splitmix64: src/Collision.h:11-16
inline uint64_t splitmix64(uint64_t& seed) {
  uint64_t z = (seed += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
struct RNGState {
  uint64_t state;
  uint64_t inc;
};
// PCG-XSH-RR 32: src/Collision.mm:21-27
inline uint32_t pcg32(RNGState& s) {
  uint64_t old = s.state;
  s.state = old * 6364136223846793005ULL + s.inc;
  uint32_t xorshifted = uint32_t(((old >> 18u) ^ old) >> 27u);
  uint32_t rot = uint32_t(old >> 59u);
  return (xorshifted >> rot) | (xorshifted << ((-rot) & 31));
}
// src/Collision.mm:28-30
inline float rand01(RNGState& s) { return float(pcg32(s)) * (1.0f / 4294967296.0f); }

// State seeding for slots [from, to): src/Collision.mm:283-294, 509-520.
inline void seed_states(std::vector<RNGState>& st, size_t from, size_t to, uint64_t& master) {
  if (st.size() < to) st.resize(to);
  for (size_t i = from; i < to; ++i) {
    uint64_t s = splitmix64(master);
    uint64_t c = splitmix64(master);
    st[i].state = s;
    st[i].inc = c | 1ULL;
  }
}

// libc++'s default_random_engine (minstd_rand, default seed 1) driving
// uniform_real_distribution<double>(0,1) through generate_canonical<double,53>
// (k = 2 draws of 30 bits). The reference's artificial-ionization count
// rounding uses a default-constructed engine member (src/Collision.mm:183,
// 476-487; the local at :298 shadows it), so on the reference's platform the
// stream is this one.
struct MinstdCanonical {
  uint64_t x = 1;
  uint64_t next() {
    x = (x * 48271ULL) % 2147483647ULL;
    return x;
  }
  double uniform01() {
    const double Rp = 2147483646.0;  // max - min + 1 for min=1, max=2^31-2
    double S = double(next() - 1);
    S += double(next() - 1) * Rp;
    return S / (Rp * Rp);
  }
};

// -------------------------------------------------------- shape factors
// Reference form, src/Particle.mm:96-131 (and :318-352, Moment.mm:78-106).
// pow(x, n) is written as repeated products.
template <typename R>
inline R p2(R a) { return a * a; }
template <typename R>
inline R p3(R a) { return a * a * a; }
template <typename R>
inline R p4(R a) { return (a * a) * (a * a); }
template <typename R>
inline R p5(R a) { return ((a * a) * (a * a)) * a; }

template <typename R>
inline void shape_ref(int order, R h, R* sf) {
  R sc;
  if (order == 1) {
    sf[0] = R(1.0) - h;
    sf[1] = h;
  } else if (order == 3) {
    const R c6 = R(1.0) / R(6.0);
    sc = R(1.0) + h;
    sf[0] = c6 * p3(R(2.0) - sc);
    sc = h;
    sf[1] = c6 * (R(4.0) - R(6.0) * p2(sc) + R(3.0) * p3(sc));
    sc = R(1.0) - h;
    sf[2] = c6 * (R(4.0) - R(6.0) * p2(sc) + R(3.0) * p3(sc));
    sc = R(2.0) - h;
    sf[3] = c6 * p3(R(2.0) - sc);
  } else if (order == 5) {
    const R c120 = R(1.0) / R(120.0);
    const R c60 = R(1.0) / R(60.0);
    sc = R(2.0) + h;
    sf[0] = c120 * p5(R(3.0) - sc);
    sc = R(1.0) + h;
    sf[1] = c120 * (R(51.0) + R(75.0) * sc - R(210.0) * p2(sc) + R(150.0) * p3(sc) - R(45.0) * p4(sc) +
                    R(5.0) * p5(sc));
    sc = h;
    sf[2] = c60 * (R(33.0) - R(30.0) * p2(sc) + R(15.0) * p4(sc) - R(5.0) * p5(sc));
    sc = R(1.0) - h;
    sf[3] = c60 * (R(33.0) - R(30.0) * p2(sc) + R(15.0) * p4(sc) - R(5.0) * p5(sc));
    sc = R(2.0) - h;
    sf[4] = c120 * (R(51.0) + R(75.0) * sc - R(210.0) * p2(sc) + R(150.0) * p3(sc) - R(45.0) * p4(sc) +
                    R(5.0) * p5(sc));
    sc = R(3.0) - h;
    sf[5] = c120 * p5(R(3.0) - sc);
  }
}

// The GPU build evaluates the same B-spline weights in Horner form around
// the particle offset h (no large cancelling terms), with fused multiply-adds.
// This restatement performs the identical FP32 operation sequence (fmaf is
// correctly rounded on both sides), so the deterministic deposit can be
// compared bit for bit.
inline void shape_build(int order, float h, float* w) {
  const float u = 1.0f - h;
  if (order == 1) {
    w[0] = u;
    w[1] = h;
  } else if (order == 3) {
    const float c6 = 1.0f / 6.0f, c23 = 2.0f / 3.0f;
    const float h2 = h * h, u2 = u * u;
    w[0] = (u2 * u) * c6;
    w[1] = std::fmaf(h2, std::fmaf(h, 0.5f, -1.0f), c23);
    w[2] = std::fmaf(u2, std::fmaf(u, 0.5f, -1.0f), c23);
    w[3] = (h2 * h) * c6;
  } else {
    const float c120 = 1.0f / 120.0f;
    const float a0 = 26.0f / 120.0f, a1 = -50.0f / 120.0f, a2 = 20.0f / 120.0f, a3 = 20.0f / 120.0f,
                a4 = -20.0f / 120.0f, a5 = 5.0f / 120.0f;
    const float b0 = 11.0f / 20.0f, b2 = -0.5f, b4 = 0.25f, b5 = -1.0f / 12.0f;
    const float h2 = h * h, u2 = u * u;
    w[0] = ((u2 * u2) * u) * c120;
    w[5] = ((h2 * h2) * h) * c120;
    // distance 1+h (and 1+u for w[4])
    w[1] = std::fmaf(h, std::fmaf(h, std::fmaf(h, std::fmaf(h, std::fmaf(h, a5, a4), a3), a2), a1), a0);
    w[4] = std::fmaf(u, std::fmaf(u, std::fmaf(u, std::fmaf(u, std::fmaf(u, a5, a4), a3), a2), a1), a0);
    // distance h (and u for w[3])
    w[2] = std::fmaf(h2, std::fmaf(h2, std::fmaf(h, b5, b4), b2), b0);
    w[3] = std::fmaf(u2, std::fmaf(u2, std::fmaf(u, b5, b4), b2), b0);
  }
}

// ---------------------------------------------------------------- grid
struct Grid {
  int ngx, ngy, ngb;
  int nx() const { return ngx + 2 * ngb; }  // src/EMField.mm:127-128
  int ny() const { return ngy + 2 * ngb; }
  size_t n_rho() const { return size_t(nx() + 1) * (ny() + 1); }
  size_t n_ex() const { return size_t(nx() + 2) * (ny() + 1); }
  size_t n_ey() const { return size_t(nx() + 1) * (ny() + 2); }
  size_t n_bz() const { return size_t(nx() + 2) * (ny() + 2); }
  size_t n_phi() const { return size_t(nx() + 3) * (ny() + 3); }
};

// ------------------------------------------------------------- particles
template <typename R>
struct Particles {
  std::vector<R> x, y, vx, vy, vz;
  std::vector<int> piflag;
  size_t n = 0;
  void resize(size_t cap) {
    x.resize(cap);
    y.resize(cap);
    vx.resize(cap);
    vy.resize(cap);
    vz.resize(cap);
    piflag.resize(cap);
  }
};

struct PushParams {
  int ngx, ngy, ngb, order, boris_order;
  int bc[4];  // Xmin, Xmax, Ymin, Ymax particle BC codes
  double constE, constB, constX, constY;
};

// Gather + Boris + position update + BCs for particle k:
// src/Particle.mm:83-269 (kernel updateParticles).
template <typename R>
inline void push_one(Particles<R>& P, size_t k, const R* Ex, const R* Ey, const R* Bz, const PushParams& prm) {
  R px = P.x[k], py = P.y[k];
  R xh = px - R(0.5);
  R yh = py - R(0.5);
  int i1 = int(std::floor(xh));
  int j1 = int(std::floor(py));
  int i2 = int(std::floor(px));
  int j2 = int(std::floor(yh));
  R hv00 = xh - R(i1), hv01 = py - R(j1), hv10 = px - R(i2), hv11 = yh - R(j2);
  R s00[6], s01[6], s10[6], s11[6];
  shape_ref<R>(prm.order, hv00, s00);
  shape_ref<R>(prm.order, hv01, s01);
  shape_ref<R>(prm.order, hv10, s10);
  shape_ref<R>(prm.order, hv11, s11);
  R Epx = 0, Epy = 0, Epz = 0, Bpx = 0, Bpy = 0, Bpz = 0;
  const int nx = prm.ngx + 2 * prm.ngb, ny = prm.ngy + 2 * prm.ngb;
  // A particle exactly on the far wall (loader draw of 1.0) reaches one node
  // past the arrays with weight 0; such taps are skipped (the reference reads
  // past its buffers there).
  auto in = [](int a, int b, int w, int h) { return a >= 0 && b >= 0 && a < w && b < h; };
  for (int i = 0; i < prm.order + 1; i++) {
    for (int j = 0; j < prm.order + 1; j++) {
      int ii = i1 + (i - prm.ngb + 1);
      int jj = j1 + (j - prm.ngb);
      if (in(ii, jj, nx + 2, ny + 1)) Epx += s00[i] * s01[j] * Ex[ii + jj * (nx + 2)];
      ii = i2 + (i - prm.ngb);
      jj = j2 + (j - prm.ngb + 1);
      if (in(ii, jj, nx + 1, ny + 2)) Epy += s10[i] * s11[j] * Ey[ii + jj * (nx + 1)];
      ii = i1 + (i - prm.ngb + 1);
      jj = j2 + (j - prm.ngb + 1);
      if (in(ii, jj, nx + 2, ny + 2)) Bpz += s00[i] * s11[j] * Bz[ii + jj * (nx + 2)];
    }
  }
  const R cE = R(prm.constE), cB = R(prm.constB);
  R etx = cE * Epx, ety = cE * Epy, etz = cE * Epz;
  R btx = cB * Bpx, bty = cB * Bpy, btz = cB * Bpz;
  R btbt = btx * btx + bty * bty + btz * btz;
  if (prm.boris_order != 2) {  // src/Particle.mm:167-186
    R fN1 = 0, fN2 = 0;
    if (prm.boris_order == 4) {
      fN1 = (R(1.0) + btbt / R(3.0));
      fN2 = R(1.0) / R(3.0);
    } else if (prm.boris_order == 6) {
      fN1 = (R(1.0) + btbt / R(3.0) + R(2.0) * btbt * btbt / R(15.0));
      fN2 = (R(1.0) / R(3.0) + R(2.0) * btbt / R(15.0));
    }
    R etbt = etx * btx + ety * bty + etz * btz;
    etx = fN1 * etx + fN2 * etbt * btx;
    ety = fN1 * ety + fN2 * etbt * bty;
    etz = fN1 * etz + fN2 * etbt * btz;
    btx = fN1 * btx;
    bty = fN1 * bty;
    btz = fN1 * btz;
  }
  R umx = P.vx[k] + etx, umy = P.vy[k] + ety, umz = P.vz[k] + etz;
  R v0x = umx + umy * btz - umz * bty;
  R v0y = umy + umz * btx - umx * btz;
  R v0z = umz + umx * bty - umy * btx;
  R ssx = R(2) * btx / (R(1) + btbt);
  R ssy = R(2) * bty / (R(1) + btbt);
  R ssz = R(2) * btz / (R(1) + btbt);
  R upx = umx + v0y * ssz - v0z * ssy;
  R upy = umy + v0z * ssx - v0x * ssz;
  R upz = umz + v0x * ssy - v0y * ssx;
  // Second half kick uses the unmodified constE*E (src/Particle.mm:207-209).
  P.vx[k] = upx + cE * Epx;
  P.vy[k] = upy + cE * Epy;
  P.vz[k] = upz + cE * Epz;
  px = px + P.vx[k] * R(prm.constX);
  py = py + P.vy[k] * R(prm.constY);
  const R fngx = R(prm.ngx), fngy = R(prm.ngy), fngb = R(prm.ngb);
  if (prm.bc[XMIN] == PBC_PERIODIC) px = std::fmod(px + R(prm.ngx - prm.ngb), fngx) + fngb;
  if (prm.bc[YMIN] == PBC_PERIODIC) py = std::fmod(py + R(prm.ngy - prm.ngb), fngy) + fngb;
  int& fl = P.piflag[k];
  if (prm.bc[XMIN] == PBC_DELETE && int(std::floor(px)) < prm.ngb) fl = 1;
  if (prm.bc[XMAX] == PBC_DELETE && int(std::floor(px)) >= prm.ngb + prm.ngx) fl = 2;
  if (prm.bc[YMIN] == PBC_DELETE && int(std::floor(py)) < prm.ngb) fl = 3;
  if (prm.bc[YMAX] == PBC_DELETE && int(std::floor(py)) >= prm.ngb + prm.ngy) fl = 4;
  if (prm.bc[XMIN] == PBC_REFLECT && int(std::floor(px)) < prm.ngb) {
    px = fngb + fngb - px;
    P.vx[k] = -P.vx[k];
  }
  if (prm.bc[XMAX] == PBC_REFLECT && int(std::floor(px)) >= prm.ngb + prm.ngx) {
    px = R(prm.ngb + prm.ngx) + R(prm.ngb + prm.ngx) - px;
    P.vx[k] = -P.vx[k];
  }
  if (prm.bc[YMIN] == PBC_REFLECT && int(std::floor(py)) < prm.ngb) {
    py = fngb + fngb - py;
    P.vy[k] = -P.vy[k];
  }
  if (prm.bc[YMAX] == PBC_REFLECT && int(std::floor(py)) >= prm.ngb + prm.ngy) {
    py = R(prm.ngb + prm.ngy) + R(prm.ngb + prm.ngy) - py;
    P.vy[k] = -P.vy[k];
  }
  P.x[k] = px;
  P.y[k] = py;
}

template <typename R>
void push_all(Particles<R>& P, const R* Ex, const R* Ey, const R* Bz, const PushParams& prm) {
#pragma omp parallel for schedule(static)
  for (long k = 0; k < long(P.n); ++k) push_one<R>(P, size_t(k), Ex, Ey, Bz, prm);
}

// Charge (and current) deposition, sequential in array order:
// src/Particle.mm:304-374 (kernel integrateChargeDensity; scale at :540).
// rho += sf*sf*scale; with current, jx += sf*sf*scale*vx, jy += ... *vy.
template <typename R>
inline void deposit_one(const Particles<R>& P, size_t k, const Grid& g, int order, R scale, bool current, R* rho,
                        R* jx, R* jy) {
  R px = P.x[k], py = P.y[k];
  R xh = px - R(0.5);
  R yh = py - R(0.5);
  int i1 = int(std::floor(xh));
  int j1 = int(std::floor(py));
  int i2 = int(std::floor(px));
  int j2 = int(std::floor(yh));
  R s00[6], s01[6], s10[6], s11[6];
  shape_ref<R>(order, xh - R(i1), s00);
  shape_ref<R>(order, py - R(j1), s01);
  shape_ref<R>(order, px - R(i2), s10);
  shape_ref<R>(order, yh - R(j2), s11);
  const int nx = g.nx(), ny = g.ny();
  auto in = [](int a, int b, int w, int h) { return a >= 0 && b >= 0 && a < w && b < h; };
  for (int i = 0; i < order + 1; i++) {
    for (int j = 0; j < order + 1; j++) {
      int ii = i2 + (i - g.ngb);
      int jj = j1 + (j - g.ngb);
      // nodes past the arrays carry weight 0 (particle exactly on the far wall)
      if (in(ii, jj, nx + 1, ny + 1)) rho[ii + jj * (nx + 1)] += s10[i] * s01[j] * scale;
      if (current) {
        ii = i1 + (i - g.ngb + 1);
        jj = j1 + (j - g.ngb);
        if (in(ii, jj, nx + 2, ny + 1)) jx[ii + jj * (nx + 2)] += s00[i] * s01[j] * scale * P.vx[k];
        ii = i2 + (i - g.ngb);
        jj = j2 + (j - g.ngb + 1);
        if (in(ii, jj, nx + 1, ny + 2)) jy[ii + jj * (nx + 1)] += s10[i] * s11[j] * scale * P.vy[k];
      }
    }
  }
}

template <typename R>
void deposit_all(const Particles<R>& P, const Grid& g, int order, R scale, bool current, R* rho, R* jx, R* jy) {
  for (size_t k = 0; k < P.n; ++k) deposit_one<R>(P, k, g, order, scale, current, rho, jx, jy);
}

// Thread-parallel deposit for the timed CPU baseline: thread-private grids
// summed in thread order (deterministic for a fixed thread count).
template <typename R>
void deposit_all_omp(const Particles<R>& P, const Grid& g, int order, R scale, bool current, R* rho, R* jx, R* jy) {
#ifdef _OPENMP
  int nt = omp_get_max_threads();
#else
  int nt = 1;
#endif
  if (nt <= 1 || P.n < 100000) {
    deposit_all<R>(P, g, order, scale, current, rho, jx, jy);
    return;
  }
  const size_t nr = g.n_rho(), nxx = g.n_ex(), nyy = g.n_ey();
  std::vector<std::vector<R>> prho(nt), pjx(nt), pjy(nt);
#pragma omp parallel num_threads(nt)
  {
#ifdef _OPENMP
    int t = omp_get_thread_num();
#else
    int t = 0;
#endif
    prho[t].assign(nr, R(0));
    if (current) {
      pjx[t].assign(nxx, R(0));
      pjy[t].assign(nyy, R(0));
    }
#pragma omp for schedule(static)
    for (long k = 0; k < long(P.n); ++k)
      deposit_one<R>(P, size_t(k), g, order, scale, current, prho[t].data(), current ? pjx[t].data() : nullptr,
                     current ? pjy[t].data() : nullptr);
  }
#pragma omp parallel for schedule(static)
  for (long i = 0; i < long(nr); ++i)
    for (int t = 0; t < nt; ++t) rho[i] += prho[t][i];
  if (current) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < long(nxx); ++i)
      for (int t = 0; t < nt; ++t) jx[i] += pjx[t][i];
#pragma omp parallel for schedule(static)
    for (long i = 0; i < long(nyy); ++i)
      for (int t = 0; t < nt; ++t) jy[i] += pjy[t][i];
  }
}

// --------------------------------------------------------------- field
// Ghost-charge folding: src/EMField.mm:751-850.
template <typename R>
void fold_ghosts(R* rho, const Grid& g, const int fbc[4]) {
  const int nx = g.nx(), ny = g.ny(), ngb = g.ngb, ngx = g.ngx, ngy = g.ngy;
  int idx_in, idx_out;
  if (fbc[XMIN] != FBC_PERIODIC) {
    for (int j = 0; j <= ny; j++) {
      if (fbc[XMIN] == FBC_DIRICHLET) {
        for (int i = 0; i <= ngb; i++) {
          idx_in = i + j * (nx + 1);
          idx_out = ngb + 1 + j * (nx + 1);
          rho[idx_out] += rho[idx_in];
        }
      } else if (fbc[XMIN] == FBC_NEUMANN) {
        for (int i = 0; i < ngb; i++) {
          idx_in = i + j * (nx + 1);
          idx_out = ngb + j * (nx + 1);
          rho[idx_out] += rho[idx_in];
        }
      }
      if (fbc[XMAX] == FBC_DIRICHLET) {
        for (int i = 0; i <= ngb; i++) {
          idx_in = ngb + ngx + i + j * (nx + 1);
          idx_out = ngb + ngx - 1 + j * (nx + 1);
          rho[idx_out] += rho[idx_in];
        }
      } else if (fbc[XMAX] == FBC_NEUMANN) {
        for (int i = 0; i < ngb; i++) {
          idx_in = ngb + ngx + i + j * (nx + 1);
          idx_out = ngb + ngx + j * (nx + 1);
          rho[idx_out] += rho[idx_in];
        }
      }
    }
  }
  if (fbc[YMIN] != FBC_PERIODIC) {
    for (int i = 0; i <= nx; i++) {
      if (fbc[YMIN] == FBC_DIRICHLET) {
        for (int j = 0; j <= ngb; j++) {
          idx_in = i + j * (nx + 1);
          idx_out = i + (ngb + 1) * (nx + 1);
          rho[idx_out] += rho[idx_in];
        }
      } else if (fbc[YMIN] == FBC_NEUMANN) {
        for (int j = 0; j < ngb; j++) {
          idx_in = i + j * (nx + 1);
          idx_out = i + (ngb) * (nx + 1);
          rho[idx_out] += rho[idx_in];
        }
      }
      if (fbc[YMAX] == FBC_DIRICHLET) {
        for (int j = 0; j <= ngb; j++) {
          idx_in = i + (ngb + ngy + j) * (nx + 1);
          idx_out = i + (ngb + ngy - 1) * (nx + 1);
          rho[idx_out] += rho[idx_in];
        }
      } else if (fbc[YMAX] == FBC_NEUMANN) {
        for (int j = 0; j < ngb; j++) {
          idx_in = i + (ngb + ngy + j) * (nx + 1);
          idx_out = i + (ngb + ngy) * (nx + 1);
          rho[idx_out] += rho[idx_in];
        }
      }
    }
  }
  if (fbc[XMIN] == FBC_PERIODIC) {
    for (int j = 0; j <= ny; j++) {
      for (int i = 0; i < ngb; i++) {
        idx_in = i + j * (nx + 1);
        idx_out = ngx + i + j * (nx + 1);
        rho[idx_out] += rho[idx_in];
      }
      for (int i = 0; i <= ngb; i++) {
        idx_in = ngb + ngx + i + j * (nx + 1);
        idx_out = ngb + i + j * (nx + 1);
        rho[idx_out] += rho[idx_in];
      }
    }
  }
  if (fbc[YMIN] == FBC_PERIODIC) {
    for (int i = 0; i <= nx; i++) {
      for (int j = 0; j < ngb; j++) {
        idx_in = i + j * (nx + 1);
        idx_out = i + (ngy + j) * (nx + 1);
        rho[idx_out] += rho[idx_in];
      }
      for (int j = 0; j <= ngb; j++) {
        idx_in = i + (ngb + ngy + j) * (nx + 1);
        idx_out = i + (ngb + j) * (nx + 1);
        rho[idx_out] += rho[idx_in];
      }
    }
  }
}

struct CSR {
  int n = 0;
  std::vector<int> ptr, col;
  std::vector<double> val;
  void matvec(const double* x, double* y) const {
#pragma omp parallel for schedule(static)
    for (int r = 0; r < n; ++r) {
      double s = 0;
      for (int k = ptr[r]; k < ptr[r + 1]; ++k) s += val[k] * x[col[k]];
      y[r] = s;
    }
  }
};

inline double dot(const std::vector<double>& a, const std::vector<double>& b) {
  double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (long i = 0; i < long(a.size()); ++i) s += a[i] * b[i];
  return s;
}

// Poisson system layout: src/EMField.mm:236-405.
struct PoissonSystem {
  Grid g;
  int fbc[4];
  double phiXmin = 0, phiXmax = 0, phiYmin = 0, phiYmax = 0;  // statV (Value * VtosV)
  double dphidxXmin = 0, dphidxXmax = 0, dphidyYmin = 0, dphidyYmax = 0;
  float dx, dy;  // src/EMField.mm:65-66 (float members)
  int nkx, ikmin, nky, jkmin;
  double Cd, Cx, Cy;
  CSR A;
  std::vector<double> rhs_BC;

  void build() {
    Cd = -2 * (1.0 / dx / dx + 1.0 / dy / dy);
    Cx = 1.0 / dx / dx;
    Cy = 1.0 / dy / dy;
    const int ngx = g.ngx, ngy = g.ngy, ngb = g.ngb;
    nkx = ngx;
    ikmin = ngb;
    if (fbc[XMIN] == FBC_DIRICHLET) {
      nkx--;
      ikmin++;
    }
    if (fbc[XMAX] == FBC_DIRICHLET) nkx--;
    if (fbc[XMIN] == FBC_PERIODIC) nkx--;
    nky = ngy;
    jkmin = ngb;
    if (fbc[YMIN] == FBC_DIRICHLET) {
      nky--;
      jkmin++;
    }
    if (fbc[YMAX] == FBC_DIRICHLET) nky--;
    if (fbc[YMIN] == FBC_PERIODIC) nky--;
    A.n = (nkx + 1) * (nky + 1);
    A.ptr.assign(1, 0);
    A.col.clear();
    A.val.clear();
    rhs_BC.clear();
    for (int j = 0; j <= nky; ++j) {
      for (int i = 0; i <= nkx; ++i) {
        int k = i + j * (nkx + 1);
        int row = 0;
        auto push = [&](int c, double v) {
          A.col.push_back(c);
          A.val.push_back(v);
          row++;
        };
        if (i == 0 && fbc[XMIN] == FBC_NEUMANN) {
          push(k, -1.0 / dx);
          push(k + 1, 1.0 / dx);
          rhs_BC.push_back(dphidxXmin);
          A.ptr.push_back(A.ptr.back() + row);
          continue;
        } else if (i == nkx && fbc[XMAX] == FBC_NEUMANN) {
          push(k, 1.0 / dx);
          push(k - 1, -1.0 / dx);
          rhs_BC.push_back(dphidxXmax);
          A.ptr.push_back(A.ptr.back() + row);
          continue;
        } else if (j == 0 && fbc[YMIN] == FBC_NEUMANN) {
          push(k, -1.0 / dy);
          push(k + (nkx + 1), 1.0 / dy);
          rhs_BC.push_back(dphidyYmin);
          A.ptr.push_back(A.ptr.back() + row);
          continue;
        } else if (j == nky && fbc[YMAX] == FBC_NEUMANN) {
          push(k, 1.0 / dx);  // src/EMField.mm:318 uses 1/dx here
          push(k - (nkx + 1), -1.0 / dx);
          rhs_BC.push_back(dphidyYmax);
          A.ptr.push_back(A.ptr.back() + row);
          continue;
        }
        push(k, Cd);
        rhs_BC.push_back(0.0);
        if (i == 0) {
          if (fbc[XMIN] == FBC_DIRICHLET)
            rhs_BC[k] += -Cx * phiXmin;
          else if (fbc[XMIN] == FBC_PERIODIC)
            push(k + nkx, Cx);
        } else {
          push(k - 1, Cx);
        }
        if (i == nkx) {
          if (fbc[XMAX] == FBC_DIRICHLET)
            rhs_BC[k] += -Cx * phiXmax;
          else if (fbc[XMAX] == FBC_PERIODIC)
            push(k - nkx, Cx);
        } else {
          push(k + 1, Cx);
        }
        if (j == 0) {
          if (fbc[YMIN] == FBC_DIRICHLET)
            rhs_BC[k] += -Cy * phiYmin;  // all entries of _phi_Ymin are equal
          else if (fbc[YMIN] == FBC_PERIODIC)
            push(k + nky * (nkx + 1), Cy);
        } else {
          push(k - (nkx + 1), Cy);
        }
        if (j == nky) {
          if (fbc[YMAX] == FBC_DIRICHLET)
            rhs_BC[k] += -Cy * phiYmax;
          else if (fbc[YMAX] == FBC_PERIODIC)
            push(k - nky * (nkx + 1), Cy);
        } else {
          push(k + (nkx + 1), Cy);
        }
        A.ptr.push_back(A.ptr.back() + row);
      }
    }
  }
  bool doubly_periodic() const { return fbc[XMIN] == FBC_PERIODIC && fbc[YMIN] == FBC_PERIODIC; }

  // rhs = rhs_BC - 4*pi*rho(i+ikmin, j+jkmin): src/EMField.mm:852-861.
  // For the doubly periodic (singular) system the build projects the rhs to
  // zero mean (reference quirk: it does not), so `project` mirrors the build.
  template <typename RF>
  std::vector<double> rhs(const RF* rho, bool project) const {
    std::vector<double> b(A.n);
    const int nx = g.nx();
    for (int j = 0; j <= nky; j++)
      for (int i = 0; i <= nkx; i++) {
        int k = i + j * (nkx + 1);
        b[k] = rhs_BC[k] - 4 * PI * static_cast<double>(rho[(i + ikmin) + (j + jkmin) * (nx + 1)]);
      }
    if (project && doubly_periodic()) {
      double m = 0;
      for (double v : b) m += v;
      m /= double(b.size());
      for (double& v : b) v -= m;
    }
    return b;
  }

  double rel_residual(const std::vector<double>& b, const std::vector<double>& x) const {
    std::vector<double> r(A.n);
    A.matvec(x.data(), r.data());
    double rr = 0, bb = 0;
    for (int i = 0; i < A.n; ++i) {
      double d = b[i] - r[i];
      rr += d * d;
      bb += b[i] * b[i];
    }
    return bb > 0 ? std::sqrt(rr / bb) : std::sqrt(rr);
  }
};

// Conjugate gradients with AMGCL's stopping rule (relative residual
// ||b - A x|| / ||b|| below tol; x cleared when ||b|| is ~0), warm-started
// from x. Returns (iterations, relative residual). Stands in for AMGCL's
// SA-AMG preconditioned CG (src/EMField.mm:20-28, 412-432, 866); AMGCL's own
// iteration path is not reproducible here.
inline std::tuple<int, double> cg_solve(const CSR& A, const std::vector<double>& b, std::vector<double>& x,
                                        double tol, int maxiter, bool zero_mean) {
  const int n = A.n;
  double norm_rhs = std::sqrt(dot(b, b));
  if (norm_rhs < std::numeric_limits<double>::epsilon()) {
    std::fill(x.begin(), x.end(), 0.0);
    return {0, norm_rhs};
  }
  std::vector<double> r(n), p(n), q(n);
  A.matvec(x.data(), q.data());
  for (int i = 0; i < n; ++i) r[i] = b[i] - q[i];
  double rho_old = 0, res = std::sqrt(dot(r, r));
  int it = 0;
  const double eps = tol * norm_rhs;
  for (; it < maxiter && res > eps; ++it) {
    double rho_new = dot(r, r);
    if (it == 0)
      p = r;
    else {
      double beta = rho_new / rho_old;
#pragma omp parallel for schedule(static)
      for (int i = 0; i < n; ++i) p[i] = r[i] + beta * p[i];
    }
    A.matvec(p.data(), q.data());
    double alpha = rho_new / dot(p, q);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
    }
    rho_old = rho_new;
    if (zero_mean && (it % 50) == 49) {  // keep the iterate in the range of A
      double m = 0;
      for (int i = 0; i < n; ++i) m += r[i];
      m /= n;
      for (int i = 0; i < n; ++i) r[i] -= m;
    }
    res = std::sqrt(dot(r, r));
  }
  if (zero_mean) {
    double m = 0;
    for (int i = 0; i < n; ++i) m += x[i];
    m /= n;
    for (int i = 0; i < n; ++i) x[i] -= m;
  }
  // true residual
  A.matvec(x.data(), q.data());
  double rr = 0;
  for (int i = 0; i < n; ++i) rr += (b[i] - q[i]) * (b[i] - q[i]);
  return {it, std::sqrt(rr) / norm_rhs};
}

// Fill the (nx+3)(ny+3) potential from the solution vector, extrapolating
// linearly into ghost nodes: src/EMField.mm:873-1061. The periodic-x index
// uses +ngx (the reference's "+ngx-1" shifts phi by one cell in x; the build
// fixes it, and `x_periodic_shift_quirk` reproduces the reference).
inline void phi_fill(const PoissonSystem& S, const std::vector<double>& sol, std::vector<double>& phi,
                     bool x_periodic_shift_quirk = false) {
  const Grid& g = S.g;
  const int nx = g.nx(), ny = g.ny(), ngb = g.ngb, ngx = g.ngx, ngy = g.ngy;
  const int nkx = S.nkx, nky = S.nky;
  phi.assign(g.n_phi(), 0.0);
  const int* fbc = S.fbc;
  auto sol_at = [&](int i, int j) { return sol[i + j * (nkx + 1)]; };
  bool isLeft = false, isRight = false, isBottom = false, isTop = false;
  int iin = 0, jin = 0;
  for (int j = 0; j <= ny + 2; ++j) {
    if (fbc[YMIN] == FBC_DIRICHLET) {
      isBottom = (j <= ngb + 1);
      jin = j - (ngb + 1) - 1;
    } else if (fbc[YMIN] == FBC_NEUMANN) {
      isBottom = (j < ngb + 1);
      jin = j - (ngb + 1);
    } else if (fbc[YMIN] == FBC_PERIODIC) {
      isBottom = false;
      isTop = false;
      jin = ((j - (ngb + 1) + ngy) % ngy + ngy) % ngy;
    }
    if (fbc[YMAX] == FBC_DIRICHLET)
      isTop = (j >= ngb + 1 + ngy);
    else if (fbc[YMAX] == FBC_NEUMANN)
      isTop = (j > ngb + 1 + ngy);
    for (int i = 0; i <= nx + 2; ++i) {
      if (fbc[XMIN] == FBC_DIRICHLET) {
        isLeft = (i <= ngb + 1);
        iin = i - (ngb + 1) - 1;
      } else if (fbc[XMIN] == FBC_NEUMANN) {
        isLeft = (i < ngb + 1);
        iin = i - (ngb + 1);
      } else if (fbc[XMIN] == FBC_PERIODIC) {
        isLeft = false;
        isRight = false;
        int sh = x_periodic_shift_quirk ? (ngx - 1) : ngx;
        iin = ((i - (ngb + 1) + sh) % ngx + ngx) % ngx;
      }
      if (fbc[XMAX] == FBC_DIRICHLET)
        isRight = (i >= ngb + 1 + ngx);
      else if (fbc[XMAX] == FBC_NEUMANN)
        isRight = (i > ngb + 1 + ngx);
      double& out = phi[i + j * (nx + 3)];
      double dphidx, dphidy;
      if (!isLeft && !isRight && !isBottom && !isTop) out = sol_at(iin, jin);
      if (isLeft && !isRight && !isBottom && !isTop) {
        if (fbc[XMIN] == FBC_DIRICHLET) {
          dphidx = sol_at(0, jin) - S.phiXmin;
          out = S.phiXmin + (i - (ngb + 1)) * dphidx;
        } else if (fbc[XMIN] == FBC_NEUMANN) {
          out = sol_at(0, jin) + (i - (ngb + 1)) * S.dphidxXmin;
        }
      }
      if (!isLeft && isRight && !isBottom && !isTop) {
        if (fbc[XMAX] == FBC_DIRICHLET) {
          dphidx = S.phiXmax - sol_at(nkx, jin);
          out = S.phiXmax + (i - (ngb + 1 + ngx)) * dphidx;
        } else if (fbc[XMAX] == FBC_NEUMANN) {
          out = sol_at(nkx, jin) + (i - (ngb + 1 + ngx)) * S.dphidxXmax;
        }
      }
      if (!isLeft && !isRight && isBottom && !isTop) {
        if (fbc[YMIN] == FBC_DIRICHLET) {
          dphidy = sol_at(iin, 0) - S.phiYmin;
          out = S.phiYmin + (j - (ngb + 1)) * dphidy;
        } else if (fbc[YMIN] == FBC_NEUMANN) {
          out = sol_at(iin, 0) + (j - (ngb + 1)) * S.dphidyYmin;
        }
      }
      if (!isLeft && !isRight && !isBottom && isTop) {
        if (fbc[YMAX] == FBC_DIRICHLET) {
          dphidy = S.phiYmax - sol_at(iin, nky);
          out = S.phiYmax + (j - (ngb + 1 + ngy)) * dphidy;
        } else if (fbc[YMAX] == FBC_NEUMANN) {
          out = sol_at(iin, nky) + (j - (ngb + 1 + ngy)) * S.dphidyYmax;
        }
      }
      // Corners (src/EMField.mm:962-1059); only reachable when both
      // directions are non-periodic.
      const int di = isLeft ? (i - (ngb + 1)) : (i - (ngb + 1 + ngx));
      const int dj = isBottom ? (j - (ngb + 1)) : (j - (ngb + 1 + ngy));
      const bool DX = isLeft ? fbc[XMIN] == FBC_DIRICHLET : fbc[XMAX] == FBC_DIRICHLET;
      const bool DY = isBottom ? fbc[YMIN] == FBC_DIRICHLET : fbc[YMAX] == FBC_DIRICHLET;
      if ((isLeft || isRight) && (isBottom || isTop) && !(isLeft && isRight) && !(isBottom && isTop)) {
        const int ci = isLeft ? 0 : nkx, cj = isBottom ? 0 : nky;
        const int ni = isLeft ? 1 : nkx - 1, nj = isBottom ? 1 : nky - 1;
        double ddx = isLeft ? (sol_at(ni, cj) - sol_at(ci, cj)) : (sol_at(ci, cj) - sol_at(ni, cj));
        double ddy = isBottom ? (sol_at(ci, nj) - sol_at(ci, cj)) : (sol_at(ci, cj) - sol_at(ci, nj));
        double nX = isLeft ? S.dphidxXmin : S.dphidxXmax;
        double nY = isBottom ? S.dphidyYmin : S.dphidyYmax;
        double base;
        if (DX && DY) {
          base = isLeft ? S.phiXmin : S.phiXmax;
        } else if (!DX && DY) {
          ddx = nX;
          base = isBottom ? S.phiYmin : S.phiYmax;
        } else if (DX && !DY) {
          ddy = nY;
          base = isLeft ? S.phiXmin : S.phiXmax;
        } else {
          ddx = nX;
          ddy = nY;
          base = sol_at(ci, cj);
        }
        out = base + di * ddx + dj * ddy;
      }
    }
  }
}

// Hollow-cathode potential shift: src/EMField.mm:1063-1077.
inline double hollow_cathode_shift(const PoissonSystem& S, const std::vector<double>& sol, std::vector<double>& phi,
                                   double cathodePos) {
  double mean = 0.0;
  if (cathodePos > 0.0) {
    const int nkx = S.nkx, nky = S.nky, nx = S.g.nx(), ny = S.g.ny(), ngb = S.g.ngb;
    for (int j = 0; j <= nky; j++) mean += sol[int(cathodePos / S.dx) + j * (nkx + 1)];
    mean /= nky + 1;
    for (int j = 0; j <= ny + 2; j++)
      for (int i = 0; i <= nx + 2; i++) phi[i + j * (nx + 3)] -= mean * ((i - ngb - 2) * S.dx) / cathodePos;
  }
  return mean;
}

// E = -grad(phi): src/EMField.mm:1080-1094 (double -> float store).
template <typename R>
void gradient(const Grid& g, float dx, float dy, const std::vector<double>& phi, R* Ex, R* Ey) {
  const int nx = g.nx(), ny = g.ny();
  for (int i = 0; i <= nx + 1; ++i)
    for (int j = 0; j <= ny; ++j)
      Ex[i + j * (nx + 2)] = R(-(phi[i + 1 + (j + 1) * (nx + 3)] - phi[i + (j + 1) * (nx + 3)]) / dx);
  for (int i = 0; i <= nx; ++i)
    for (int j = 0; j <= ny + 1; ++j)
      Ey[i + j * (nx + 1)] = R(-(phi[i + 1 + (j + 1) * (nx + 3)] - phi[i + 1 + (j)*(nx + 3)]) / dy);
}

// Field energy and Joule heating: src/EMField.mm:1096-1113.
template <typename R>
void field_energy(const Grid& g, float dx, float dy, double dt, const R* Ex, const R* Ey, const R* jx, const R* jy,
                  double& energy, double& joule) {
  energy = 0;
  joule = 0;
  for (size_t i = 0; i < g.n_ex(); i++) {
    energy += double(Ex[i]) * Ex[i];
    joule += double(Ex[i]) * jx[i];
  }
  for (size_t i = 0; i < g.n_ey(); i++) {
    energy += double(Ey[i]) * Ey[i];
    joule += double(Ey[i]) * jy[i];
  }
  energy *= double(dx) * dy / 2;
  joule *= double(dt) * dx * dy;
}

// ------------------------------------------------------- compaction
struct FlowStats {
  int pinum[4] = {0, 0, 0, 0};
  int pulled = 0;
  double energy = 0;
};

// In-place removal of flagged particles, filling holes from the tail:
// src/Particle.mm:893-968. With `faithful`, the reference's extra pull when a
// tail scan runs out of live particles (it re-counts the next, already
// scanned, dead slot: :908-925 after :942-964) is reproduced; without it every
// flagged particle is counted exactly once. When every particle is flagged
// the tail scan has pulled all n and there is no slot left to re-count (the
// reference would pull n + 1 and underflow pNum): the extra pull is skipped.
template <typename R>
FlowStats reduce_particles(Particles<R>& P, float q, bool faithful) {
  FlowStats fs;
  const int unit = int(q / float(ec));
  auto count = [&](int fl) {
    if (fl >= 1 && fl <= 4) fs.pinum[fl - 1] += unit;
  };
  int n = int(P.n);
  int kmax = n, pulln = 0;
  auto copy = [&](int dst, int src) {
    P.x[dst] = P.x[src];
    P.y[dst] = P.y[src];
    P.vx[dst] = P.vx[src];
    P.vy[dst] = P.vy[src];
    P.vz[dst] = P.vz[src];
    P.piflag[dst] = P.piflag[src];
  };
  for (int k1 = 0; k1 < n; k1++) {
    if (k1 >= kmax) {
      if (faithful && P.piflag[k1] > 0 && pulln < n) {
        pulln++;
        count(P.piflag[k1]);
      }
      break;
    }
    if (P.piflag[k1] > 0) {
      count(P.piflag[k1]);
      int kend = kmax;
      for (int k2 = kend - 1; k2 >= k1; k2--) {
        kmax--;
        pulln++;
        if (P.piflag[k2] == 0) {
          copy(k1, k2);
          break;
        }
        if (k2 > k1) count(P.piflag[k2]);
      }
    }
  }
  fs.pulled = pulln;
  P.n = size_t(n - pulln);
  return fs;
}

// Kinetic energy of the live particles: src/Particle.mm:970-984 (v*v summed
// in float, promoted to double).
template <typename R>
double kinetic_energy(const Particles<R>& P, float m, float w) {
  double energy = 0.0;
  for (size_t k = 0; k < P.n; ++k) {
    R vvf = P.vx[k] * P.vx[k] + P.vy[k] * P.vy[k] + P.vz[k] * P.vz[k];
    double vv = double(vvf);
    energy += double(0.5 * double(m) * vv * double(w));
  }
  return energy;
}

// ------------------------------------------------------ generation
// Parameters of kernel artificialIonization (src/Collision.h:22-38).
struct GenParams {
  uint32_t addn = 0, ele_pNum = 0, ion_pNum = 0;
  float Xmin = 0, Xmax = 0, Ymin = 0, Ymax = 0;
  float ele_genU[3] = {0, 0, 0};
  float ele_vth = 0;
  float ion_genU[3] = {0, 0, 0};
  float ion_vth = 0;
  float dx = 0, dy = 0, ngb = 0;
};

// One new particle (pair): src/Collision.mm:70-173. genType 0 uniform,
// 1 X-sinusoidal, 2 Y-sinusoidal, 3 hollow-cathode (electron only),
// 4 quiet start, 5 X-Gaussian, 6 Y-Gaussian.
template <typename R>
inline void generate_one(uint32_t id, int genType, const GenParams& prm, RNGState* states, Particles<R>& ele,
                         Particles<R>* ion) {
  RNGState rng = states[id];
  const float fPI = float(PI);
  float ex = 0, ey = 0;
  float rx = rand01(rng);
  float ry = rand01(rng);
  if (genType == 0 || genType == 3) {
    ex = prm.Xmin + rx * (prm.Xmax - prm.Xmin);
    ey = prm.Ymin + ry * (prm.Ymax - prm.Ymin);
  } else if (genType == 1) {
    ex = (prm.Xmin + prm.Xmax) / 2 + (prm.Xmax - prm.Xmin) / fPI * std::asin(2 * rx - 1.0f);
    ey = prm.Ymin + ry * (prm.Ymax - prm.Ymin);
  } else if (genType == 2) {
    ex = prm.Xmin + rx * (prm.Xmax - prm.Xmin);
    ey = (prm.Ymin + prm.Ymax) / 2 + (prm.Ymax - prm.Ymin) / fPI * std::asin(2 * ry - 1.0f);
  } else if (genType == 4) {
    int addn_x = int(std::round(std::sqrt(float(prm.addn) * (prm.Xmax - prm.Xmin) / (prm.Ymax - prm.Ymin))));
    int addn_y = int(prm.addn) / addn_x;
    float delta_x = (prm.Xmax - prm.Xmin) / addn_x;
    float delta_y = (prm.Ymax - prm.Ymin) / addn_y;
    ex = prm.Xmin + delta_x * (0.5f + float(id % uint32_t(addn_x)));
    ey = prm.Ymin + delta_y * (0.5f + float(id / uint32_t(addn_x)));
  } else if (genType == 5) {
    float rz = rand01(rng);
    ex = (prm.Xmin + prm.Xmax) / 2 + (prm.Xmax - prm.Xmin) * std::sqrt(-std::log(rx)) * std::cos(2.0f * fPI * rz);
    ey = prm.Ymin + ry * (prm.Ymax - prm.Ymin);
  } else if (genType == 6) {
    float rz = rand01(rng);
    ex = prm.Xmin + rx * (prm.Xmax - prm.Xmin);
    ey = (prm.Ymin + prm.Ymax) / 2 + (prm.Ymax - prm.Ymin) * std::sqrt(-std::log(rz)) * std::cos(2.0f * fPI * ry);
  }
  float rv1 = rand01(rng), rv2 = rand01(rng);
  float evx = prm.ele_genU[0] + prm.ele_vth * std::sqrt(-std::log(rv1)) * std::cos(2.0f * fPI * rv2);
  float evy = prm.ele_genU[1] + prm.ele_vth * std::sqrt(-std::log(rv1)) * std::sin(2.0f * fPI * rv2);
  rv1 = rand01(rng);
  rv2 = rand01(rng);
  float evz = prm.ele_genU[2] + prm.ele_vth * std::sqrt(-std::log(rv1)) * std::cos(2.0f * fPI * rv2);
  ex = ex / prm.dx;
  ey = ey / prm.dy;
  ex = ex + prm.ngb;
  ey = ey + prm.ngb;
  size_t ke = prm.ele_pNum + id;
  ele.x[ke] = R(ex);
  ele.y[ke] = R(ey);
  ele.vx[ke] = R(evx);
  ele.vy[ke] = R(evy);
  ele.vz[ke] = R(evz);
  ele.piflag[ke] = 0;
  if (genType != 3 && ion) {
    size_t ki = prm.ion_pNum + id;
    ion->x[ki] = R(ex);
    ion->y[ki] = R(ey);
    rv1 = rand01(rng);
    rv2 = rand01(rng);
    ion->vx[ki] = R(prm.ion_genU[0] + prm.ion_vth * std::sqrt(-std::log(rv1)) * std::cos(2.0f * fPI * rv2));
    ion->vy[ki] = R(prm.ion_genU[1] + prm.ion_vth * std::sqrt(-std::log(rv1)) * std::sin(2.0f * fPI * rv2));
    rv1 = rand01(rng);
    rv2 = rand01(rng);
    ion->vz[ki] = R(prm.ion_genU[2] + prm.ion_vth * std::sqrt(-std::log(rv1)) * std::cos(2.0f * fPI * rv2));
    ion->piflag[ki] = 0;
  }
  states[id] = rng;
}

// -------------------------------------------------------- Darwin model
// src/EMField.mm:447-651 (operator) and 1138-1361 (solveVectorPotential) on
// the vector-potential grid (nkx+1)(nky+1), nkx = ngx - [x periodic]. The
// build's documented choices are restated too: with a Neumann direction the
// right-hand side is also projected with the solvability weights (1/2 at
// the ends), solutions have zero mean, the last column (row) of a periodic
// direction closes through the wrap, and delEy sits at (i+ngb, j+ngb+1).
// Solves: CG on the symmetrised operator W A (W = the weights) to 1e-13.
struct DarwinIn {
  int ngx, ngy, ngb;
  bool perx, pery;
  float dx, dy;
  double dt;
};

inline double darwin_weight(int i, int n, bool per) { return (!per && (i == 0 || i == n - 1)) ? 0.5 : 1.0; }

inline CSR darwin_csr(int nkx, int nky, bool perx, bool pery, double Cx, double Cy, double Cd, bool symmetrise) {
  CSR A;
  const int mx = nkx + 1, my = nky + 1;
  A.n = mx * my;
  A.ptr.push_back(0);
  for (int j = 0; j < my; ++j)
    for (int i = 0; i < mx; ++i) {
      const int k = i + j * mx;
      const double w = symmetrise ? darwin_weight(i, mx, perx) * darwin_weight(j, my, pery) : 1.0;
      std::vector<std::pair<int, double>> e;
      e.push_back({k, Cd});
      auto side = [&](int idx, int n, bool per, int stride, double C) {
        if (idx == 0) {
          if (per) {
            e.push_back({k + (n - 1) * stride, C});
            e.push_back({k + stride, C});
          } else if (n > 1) {
            e.push_back({k + stride, 2 * C});  // Neumann: doubled off-diagonal (src/EMField.mm:531-537)
          }
        } else if (idx == n - 1) {
          if (per) {
            e.push_back({k - stride, C});
            e.push_back({k - (n - 1) * stride, C});
          } else {
            e.push_back({k - stride, 2 * C});
          }
        } else {
          e.push_back({k - stride, C});
          e.push_back({k + stride, C});
        }
      };
      side(i, mx, perx, 1, Cx);
      side(j, my, pery, mx, Cy);
      for (auto& q : e) {
        A.col.push_back(q.first);
        A.val.push_back(w * q.second);
      }
      A.ptr.push_back(int(A.col.size()));
    }
  return A;
}

template <typename R>
void darwin_solve(const DarwinIn& in, const R* jx, const R* jy, std::vector<double>& psi, std::vector<double>& Ax,
                  std::vector<double>& Ay, std::vector<double>& lastAx, std::vector<double>& lastAy, float* delEx,
                  float* delEy, float* delBz) {
  const int nkx = in.ngx - (in.perx ? 1 : 0), nky = in.ngy - (in.pery ? 1 : 0);
  const int mx = nkx + 1, my = nky + 1, n = mx * my;
  const int ngb = in.ngb, nx = in.ngx + 2 * ngb;
  const float dx = in.dx, dy = in.dy;
  const double Cx = 1.0 / dx / dx, Cy = 1.0 / dy / dy, Cd = -2 * (1.0 / dx / dx + 1.0 / dy / dy);
  const CSR WA = darwin_csr(nkx, nky, in.perx, in.pery, Cx, Cy, Cd, true);
  auto solve = [&](std::vector<double> rhs, std::vector<double>& x) {
    double m = 0;
    for (double v : rhs) m += v;
    m /= n;
    for (double& v : rhs) v -= m;  // src/EMField.mm:1186-1191
    double sw = 0, ww = 0;
    for (int k = 0; k < n; ++k) {
      const double w = darwin_weight(k % mx, mx, in.perx) * darwin_weight(k / mx, my, in.pery);
      sw += w * rhs[k];
      ww += w;
    }
    for (double& v : rhs) v -= sw / ww;
    std::vector<double> wb(n);
    for (int k = 0; k < n; ++k) wb[k] = darwin_weight(k % mx, mx, in.perx) * darwin_weight(k / mx, my, in.pery) * rhs[k];
    x.assign(n, 0.0);
    cg_solve(WA, wb, x, 1e-13, 20000, true);
    double xm = 0;
    for (double v : x) xm += v;
    xm /= n;
    for (double& v : x) v -= xm;
  };
  // div J (src/EMField.mm:1150-1184)
  std::vector<double> rhs(n);
  for (int j = 0; j <= nky; j++)
    for (int i = 0; i <= nkx; i++) {
      double r = 0.0;
      const int ix = i + ngb, iy = j + ngb;
      if (!in.perx) {
        if (i == 0)
          r += double(-2 * float(jx[ix + iy * (nx + 2)]) / dx);
        else if (i == nkx)
          r += double(2 * float(jx[ix + iy * (nx + 2)]) / dx);
      }
      if (!in.pery) {
        if (j == 0)
          r += double(-2 * float(jy[ix + iy * (nx + 1)]) / dy);
        else if (j == nky)
          r += double(2 * float(jy[ix + iy * (nx + 1)]) / dy);
      }
      const double djx = double((float(jx[ix + 1 + iy * (nx + 2)]) - float(jx[ix + iy * (nx + 2)])) / dx);
      const double djy = double((float(jy[ix + (iy + 1) * (nx + 1)]) - float(jy[ix + iy * (nx + 1)])) / dy);
      rhs[i + j * mx] = r + (djx + djy);
    }
  solve(rhs, psi);
  const double f = -4 * PI / 2.99792458e10;
  for (int j = 0; j <= nky; j++)  // src/EMField.mm:1201-1229
    for (int i = 0; i <= nkx; i++) {
      const int k = i + j * mx;
      double r = 0.0;
      if (i < nkx || in.perx) {
        const int k1 = i < nkx ? k + 1 : k - nkx;
        const double jl = (psi[k1] - psi[k]) / double(dx);
        r = f * (double(float(jx[(i + ngb + 1) + (j + ngb) * (nx + 2)])) - jl);
      }
      rhs[k] = r;
    }
  solve(rhs, Ax);
  for (int j = 0; j <= nky; j++)  // src/EMField.mm:1239-1267
    for (int i = 0; i <= nkx; i++) {
      const int k = i + j * mx;
      double r = 0.0;
      if (j < nky || in.pery) {
        const int k1 = j < nky ? k + mx : k - nky * mx;
        const double jl = (psi[k1] - psi[k]) / double(dy);
        r = f * (double(float(jy[(i + ngb) + (j + ngb + 1) * (nx + 1)])) - jl);
      }
      rhs[k] = r;
    }
  solve(rhs, Ay);
  const double cdt = 2.99792458e10 * in.dt;  // src/EMField.mm:1277-1297
  const int ni = in.perx ? nkx + 1 : nkx, nj = in.pery ? nky + 1 : nky;
  for (int j = 0; j < nj; j++)
    for (int i = 0; i < ni; i++) {
      const int kf = i + j * mx;
      const int kx1 = i < nkx ? kf + 1 : kf - nkx, ky1 = j < nky ? kf + mx : kf - nky * mx;
      const int kpx = (i + ngb + 1) + (j + ngb) * (nx + 2);
      const int kpy = (i + ngb) + (j + ngb + 1) * (nx + 1);
      delEx[kpx] = float(-(Ax[kf] - lastAx[kf]) / cdt);
      delEy[kpy] = float(-(Ay[kf] - lastAy[kf]) / cdt);
      delBz[kpx + (nx + 2)] = float((Ay[kx1] - Ay[kf]) / double(dx) - (Ax[ky1] - Ax[kf]) / double(dy));
    }
  lastAx = Ax;
  lastAy = Ay;
}

// -------------------------------------------------------- moments
// Velocity moments of one species: src/Moment.mm:55-129 (kernel) and
// :287-316 (normalisation). Outputs 10 arrays of (nx+1)(ny+1):
// n, ux, uy, uz, Pxx, Pxy, Pxz, Pyy, Pyz, Pzz.
// build = true: Horner-form weights (shape_build) and FP64 sums, the
// summation the GPU build performs (for parity checks); false: the
// reference's pow-form weights and FP32 sums.
template <typename R>
void moments(const Particles<R>& P, const Grid& g, int order, float scale, float m, std::vector<float>* out,
             bool build = false) {
  const int nx = g.nx();
  const size_t ng = g.n_rho();
  for (int a = 0; a < 10; ++a) out[a].assign(ng, 0.0f);
  std::vector<double> sum(build ? 10 * ng : 0, 0.0);
  for (size_t k = 0; k < P.n; ++k) {
    if (P.piflag[k] != 0) continue;
    float px = float(P.x[k]), py = float(P.y[k]);
    int i1 = int(px + 1e-20f), j1 = int(py + 1e-20f);
    float sx[6], sy[6];
    if (build) {
      shape_build(order, px - float(i1), sx);
      shape_build(order, py - float(j1), sy);
    } else {
      shape_ref<float>(order, px - float(i1), sx);
      shape_ref<float>(order, py - float(j1), sy);
    }
    float vx = float(P.vx[k]), vy = float(P.vy[k]), vz = float(P.vz[k]);
    for (int i = 0; i < order + 1; i++)
      for (int j = 0; j < order + 1; j++) {
        const int ii = i1 + (i - g.ngb), jj = j1 + (j - g.ngb);
        if (ii < 0 || jj < 0 || ii > nx || jj > g.ny()) continue;
        int idx = ii + jj * (nx + 1);
        float s = sx[i] * sy[j];
        const float v[10] = {s * scale,   s * vx,      s * vy,      s * vz,      s * vx * vx,
                             s * vx * vy, s * vx * vz, s * vy * vy, s * vy * vz, s * vz * vz};
        if (build)
          for (int a = 0; a < 10; ++a) sum[a * ng + idx] += double(v[a]);
        else
          for (int a = 0; a < 10; ++a) out[a][idx] += v[a];
      }
  }
  if (build)
    for (int a = 0; a < 10; ++a)
      for (size_t i = 0; i < ng; ++i) out[a][i] = float(sum[a * ng + i]);
  for (size_t i = 0; i < ng; i++) {
    float n = out[0][i];
    if (n > 1e-20f) {
      out[1][i] /= n / scale;
      out[2][i] /= n / scale;
      out[3][i] /= n / scale;
    } else {
      out[1][i] = out[2][i] = out[3][i] = 0.0f;
    }
  }
  for (size_t i = 0; i < ng; i++) {
    float n = out[0][i];
    float ux = out[1][i], uy = out[2][i], uz = out[3][i];
    if (n > 1e-20f) {
      out[4][i] = m * (out[4][i] / (n / scale) - ux * ux) * n;
      out[5][i] = m * (out[5][i] / (n / scale) - ux * uy) * n;
      out[6][i] = m * (out[6][i] / (n / scale) - ux * uz) * n;
      out[7][i] = m * (out[7][i] / (n / scale) - uy * uy) * n;
      out[8][i] = m * (out[8][i] / (n / scale) - uy * uz) * n;
      out[9][i] = m * (out[9][i] / (n / scale) - uz * uz) * n;
    } else {
      for (int a = 4; a < 10; ++a) out[a][i] = 0.0f;
    }
  }
}

}  // namespace oracle
