// generate_kernels.cu -- particle loading and injection (sm_100a).
//
// Restates kernel artificialIonization (src/Collision.mm:63-174): one thread
// per new particle (pair), a persistent PCG-XSH-RR 32 state per slot
// (src/Collision.mm:21-30) seeded by splitmix64 (src/Collision.h:11-16,
// src/Collision.mm:283-294). Position arithmetic uses explicitly rounded
// float operations so the loaded positions equal the reference's FP32 values
// bit for bit; transcendental functions are CUDA's accurate (non-fast-math)
// versions.
#include <cuda_runtime.h>

#include "device.hpp"
#include "pdl.cuh"
#include "kernels.hpp"
#include "pic_common.cuh"

namespace gample {
namespace kern {

namespace {

__device__ __forceinline__ unsigned long long splitmix_at(unsigned long long seed0, unsigned long long k) {
  // k-th output (k >= 1) of splitmix64 started from seed0.
  unsigned long long z = seed0 + k * 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

__device__ __forceinline__ uint32_t pcg32(RNGState& s) {
  const unsigned long long old = s.state;
  s.state = old * 6364136223846793005ULL + s.inc;
  const uint32_t xorshifted = uint32_t(((old >> 18u) ^ old) >> 27u);
  const uint32_t rot = uint32_t(old >> 59u);
  return (xorshifted >> rot) | (xorshifted << ((0u - rot) & 31u));
}
__device__ __forceinline__ float rand01(RNGState& s) { return __fmul_rn(float(pcg32(s)), 1.0f / 4294967296.0f); }

__global__ void k_seed(RNGState* st, unsigned long long seed0, uint32_t from, uint32_t to) {
  for (uint32_t i = from + blockIdx.x * blockDim.x + threadIdx.x; i < to; i += gridDim.x * blockDim.x) {
    RNGState r;
    r.state = splitmix_at(seed0, 2ULL * i + 1ULL);
    r.inc = splitmix_at(seed0, 2ULL * i + 2ULL) | 1ULL;
    st[i] = r;
  }
}

// Convert a physical position (cm) to (cell, offset) exactly as the
// reference's x/dx + ngb in float (src/Collision.mm:122-128).
__device__ __forceinline__ bool to_cell(float xphys, float d, float ngb, int& i, float& o) {
  const float x = __fadd_rn(__fdiv_rn(xphys, d), ngb);
  if (!isfinite(x) || x < 0.0f || x >= 32767.0f) return false;
  const float fl = floorf(x);
  i = int(fl);
  o = __fsub_rn(x, fl);
  return true;
}

__device__ __forceinline__ float maxwell(float u, float vth, float r1, float r2, bool use_sin) {
  const float twoPI = 2.0f * 3.141592653589793f;
  const float a = __fmul_rn(vth, sqrtf(-logf(r1)));
  const float ang = __fmul_rn(twoPI, r2);
  return __fadd_rn(u, __fmul_rn(a, use_sin ? sinf(ang) : cosf(ang)));
}

__device__ __forceinline__ void store(ParticleArrays p, uint32_t k, bool ok, int ix, float ox, int iy, float oy,
                                      float vx, float vy, float vz) {
  p.cell[k] = ok ? pack_cell(ix, iy) : -5;
  p.ox[k] = ok ? ox : 0.0f;
  p.oy[k] = ok ? oy : 0.0f;
  p.vx[k] = vx;
  p.vy[k] = vy;
  p.vz[k] = vz;
}

template <int GT>
__global__ void k_generate(uint32_t addn, GenParams prm, RNGState* states, ParticleArrays ele,
                           const SpeciesCounters* ecnt, ParticleArrays ion, const SpeciesCounters* icnt,
                           bool with_ion) {
  grid_dependency_wait();
  grid_dependents_launch();
  const uint32_t ebase = ecnt->n;
  const uint32_t ibase = with_ion ? icnt->n : 0u;
  const float PIf = 3.141592653589793f;
  for (uint32_t id = blockIdx.x * blockDim.x + threadIdx.x; id < addn; id += gridDim.x * blockDim.x) {
    RNGState rng = states[id];
    const float rx = rand01(rng);
    const float ry = rand01(rng);
    const float Lx = __fsub_rn(prm.Xmax, prm.Xmin), Ly = __fsub_rn(prm.Ymax, prm.Ymin);
    float x = 0.0f, y = 0.0f;
    if constexpr (GT == 0 || GT == 3) {
      x = __fadd_rn(prm.Xmin, __fmul_rn(rx, Lx));
      y = __fadd_rn(prm.Ymin, __fmul_rn(ry, Ly));
    } else if constexpr (GT == 1) {
      x = __fadd_rn(__fdiv_rn(__fadd_rn(prm.Xmin, prm.Xmax), 2.0f),
                    __fmul_rn(__fdiv_rn(Lx, PIf), asinf(__fsub_rn(__fmul_rn(2.0f, rx), 1.0f))));
      y = __fadd_rn(prm.Ymin, __fmul_rn(ry, Ly));
    } else if constexpr (GT == 2) {
      x = __fadd_rn(prm.Xmin, __fmul_rn(rx, Lx));
      y = __fadd_rn(__fdiv_rn(__fadd_rn(prm.Ymin, prm.Ymax), 2.0f),
                    __fmul_rn(__fdiv_rn(Ly, PIf), asinf(__fsub_rn(__fmul_rn(2.0f, ry), 1.0f))));
    } else if constexpr (GT == 4) {
      const int addn_x = int(roundf(sqrtf(__fdiv_rn(__fmul_rn(float(addn), Lx), Ly))));
      const int addn_y = int(addn) / (addn_x > 0 ? addn_x : 1);
      const float delta_x = __fdiv_rn(Lx, float(addn_x)), delta_y = __fdiv_rn(Ly, float(addn_y));
      x = __fadd_rn(prm.Xmin, __fmul_rn(delta_x, __fadd_rn(0.5f, float(id % uint32_t(addn_x)))));
      y = __fadd_rn(prm.Ymin, __fmul_rn(delta_y, __fadd_rn(0.5f, float(id / uint32_t(addn_x)))));
    } else if constexpr (GT == 5) {
      const float rz = rand01(rng);
      x = __fadd_rn(__fdiv_rn(__fadd_rn(prm.Xmin, prm.Xmax), 2.0f),
                    __fmul_rn(__fmul_rn(Lx, sqrtf(-logf(rx))), cosf(__fmul_rn(2.0f * PIf, rz))));
      y = __fadd_rn(prm.Ymin, __fmul_rn(ry, Ly));
    } else if constexpr (GT == 6) {
      const float rz = rand01(rng);
      x = __fadd_rn(prm.Xmin, __fmul_rn(rx, Lx));
      y = __fadd_rn(__fdiv_rn(__fadd_rn(prm.Ymin, prm.Ymax), 2.0f),
                    __fmul_rn(__fmul_rn(Ly, sqrtf(-logf(rz))), cosf(__fmul_rn(2.0f * PIf, ry))));
    }
    float rv1 = rand01(rng), rv2 = rand01(rng);
    float evx = maxwell(prm.ele_genU[0], prm.ele_vth, rv1, rv2, false);
    float evy = maxwell(prm.ele_genU[1], prm.ele_vth, rv1, rv2, true);
    rv1 = rand01(rng);
    rv2 = rand01(rng);
    float evz = maxwell(prm.ele_genU[2], prm.ele_vth, rv1, rv2, false);
    float ph = 0.0f;  // drift profile of the build-added sinusoidal drift
    if (prm.sin_on) ph = sinf(__fmul_rn(2.0f * PIf, __fdiv_rn(__fsub_rn(x, prm.Xmin), Lx)));
    if (prm.sin_on) {
      evx = __fmaf_rn(prm.ele_sinU[0], ph, evx);
      evy = __fmaf_rn(prm.ele_sinU[1], ph, evy);
      evz = __fmaf_rn(prm.ele_sinU[2], ph, evz);
    }
    int ix = 0, iy = 0;
    float ox = 0.0f, oy = 0.0f;
    const bool ok = to_cell(x, prm.dx, prm.ngb, ix, ox) & to_cell(y, prm.dy, prm.ngb, iy, oy);
    store(ele, ebase + id, ok, ix, ox, iy, oy, evx, evy, evz);
    if (GT != 3 && with_ion) {
      rv1 = rand01(rng);
      rv2 = rand01(rng);
      float ivx = maxwell(prm.ion_genU[0], prm.ion_vth, rv1, rv2, false);
      float ivy = maxwell(prm.ion_genU[1], prm.ion_vth, rv1, rv2, true);
      rv1 = rand01(rng);
      rv2 = rand01(rng);
      float ivz = maxwell(prm.ion_genU[2], prm.ion_vth, rv1, rv2, false);
      if (prm.sin_on) {
        ivx = __fmaf_rn(prm.ion_sinU[0], ph, ivx);
        ivy = __fmaf_rn(prm.ion_sinU[1], ph, ivy);
        ivz = __fmaf_rn(prm.ion_sinU[2], ph, ivz);
      }
      store(ion, ibase + id, ok, ix, ox, iy, oy, ivx, ivy, ivz);
    }
    states[id] = rng;
  }
}

__global__ void k_advance_counts(SpeciesCounters* a, SpeciesCounters* b, uint32_t addn) {
  grid_dependency_wait();
  grid_dependents_launch();
  a->n += addn;
  a->n_injected += addn;
  if (b) {
    b->n += addn;
    b->n_injected += addn;
  }
}

__global__ void k_reflux(uint32_t addn, RefluxParams prm, RNGState* states, ParticleArrays p,
                         const SpeciesCounters* cnt) {
  grid_dependency_wait();
  grid_dependents_launch();
  const uint32_t base = cnt->n;
  const float twoPI = 2.0f * 3.141592653589793f;
  for (uint32_t id = blockIdx.x * blockDim.x + threadIdx.x; id < addn; id += gridDim.x * blockDim.x) {
    RNGState rng = states[id];
    const float r1 = rand01(rng), r2 = rand01(rng), r3 = rand01(rng), r4 = rand01(rng), r5 = rand01(rng);
    const float vx = __fadd_rn(prm.u0, __fmul_rn(prm.vth, sqrtf(-logf(r1))));
    const float a = __fmul_rn(prm.vth, sqrtf(-logf(r2)));
    const float ang = __fmul_rn(twoPI, r3);
    const float vy = __fadd_rn(prm.u1, __fmul_rn(a, cosf(ang)));
    const float vz = __fadd_rn(prm.u2, __fmul_rn(a, sinf(ang)));
    const float x = __fadd_rn(prm.Xmin, __fmul_rn(r5, __fmul_rn(vx, prm.dt)));
    const float y = __fadd_rn(prm.Ymin, __fmul_rn(r4, __fsub_rn(prm.Ymax, prm.Ymin)));
    int ix = 0, iy = 0;
    float ox = 0.0f, oy = 0.0f;
    const bool ok = to_cell(x, prm.dx, prm.ngb, ix, ox) & to_cell(y, prm.dy, prm.ngb, iy, oy);
    store(p, base + id, ok, ix, ox, iy, oy, vx, vy, vz);
    states[id] = rng;
  }
}

int gen_grid(uint32_t n) {
  long long b = ((long long)n + 255) / 256;
  return int(b < 4096 ? (b < 1 ? 1 : b) : 4096);
}

}  // namespace

void seed_rng(RNGState* states, uint64_t master_seed, uint32_t from, uint32_t to, cudaStream_t s) {
  if (to <= from) return;
  k_seed<<<gen_grid(to - from), 256, 0, s>>>(states, master_seed, from, to);
  GP_LAUNCH_CHECK();
}

void generate(int gen_type, uint32_t addn, GenParams prm, RNGState* states, ParticleArrays ele,
              SpeciesCounters* ecnt, ParticleArrays* ion, SpeciesCounters* icnt, cudaStream_t s) {
  if (addn == 0) return;
  const bool with_ion = ion != nullptr && gen_type != 3;
  ParticleArrays ia = with_ion ? *ion : ele;
  const SpeciesCounters* ic = with_ion ? icnt : ecnt;
  const int grid = gen_grid(addn);
#define GP_GEN(T) \
  launch_pdl(k_generate<T>, dim3(grid), dim3(256), 0, s, addn, prm, states, ele, ecnt, ia, ic, with_ion)
  switch (gen_type) {
    case 0: GP_GEN(0); break;
    case 1: GP_GEN(1); break;
    case 2: GP_GEN(2); break;
    case 3: GP_GEN(3); break;
    case 4: GP_GEN(4); break;
    case 5: GP_GEN(5); break;
    case 6: GP_GEN(6); break;
    default: throw std::invalid_argument("unknown GenerateType");
  }
#undef GP_GEN
  launch_pdl(k_advance_counts, dim3(1), dim3(1), 0, s, ecnt, with_ion ? icnt : nullptr, addn);
}

void reflux(uint32_t addn, RefluxParams prm, RNGState* states, ParticleArrays p, SpeciesCounters* cnt,
            cudaStream_t s) {
  if (addn == 0) return;
  launch_pdl(k_reflux, dim3(gen_grid(addn)), dim3(256), 0, s, addn, prm, states, p, cnt);
  launch_pdl(k_advance_counts, dim3(1), dim3(1), 0, s, cnt, nullptr, addn);
}

}  // namespace kern
}  // namespace gample
