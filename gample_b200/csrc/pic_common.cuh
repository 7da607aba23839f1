// pic_common.cuh -- device helpers shared by the particle kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.hpp"

namespace gample {
namespace kern {

constexpr float kQuant = 1099511627776.0f;  // 2^40: fixed-point scale of the deterministic deposit

__device__ __forceinline__ int cell_ix(int32_t c) { return c & 0xFFFF; }
__device__ __forceinline__ int cell_iy(int32_t c) { return c >> 16; }
__device__ __forceinline__ int32_t pack_cell(int ix, int iy) { return (iy << 16) | ix; }

// Linear/cubic/quintic B-spline weights of a particle at offset h in [0,1)
// from the stencil base (stencil nodes base-ngb .. base-ngb+ORDER), i.e. the
// reference's sf[0..ORDER] (src/Particle.mm:96-131) evaluated in Horner form
// around h. Every operation is an explicitly rounded intrinsic so that a CPU
// restatement with fmaf() reproduces the weights bit for bit.
template <int ORDER>
__device__ __forceinline__ void shape(float h, float (&w)[ORDER + 1]) {
  const float u = __fsub_rn(1.0f, h);
  if constexpr (ORDER == 1) {
    w[0] = u;
    w[1] = h;
  } else if constexpr (ORDER == 3) {
    constexpr float c6 = 1.0f / 6.0f, c23 = 2.0f / 3.0f;
    const float h2 = __fmul_rn(h, h), u2 = __fmul_rn(u, u);
    w[0] = __fmul_rn(__fmul_rn(u2, u), c6);
    w[1] = __fmaf_rn(h2, __fmaf_rn(h, 0.5f, -1.0f), c23);
    w[2] = __fmaf_rn(u2, __fmaf_rn(u, 0.5f, -1.0f), c23);
    w[3] = __fmul_rn(__fmul_rn(h2, h), c6);
  } else {
    constexpr float c120 = 1.0f / 120.0f;
    constexpr float a0 = 26.0f / 120.0f, a1 = -50.0f / 120.0f, a2 = 20.0f / 120.0f, a3 = 20.0f / 120.0f,
                    a4 = -20.0f / 120.0f, a5 = 5.0f / 120.0f;
    constexpr float b0 = 11.0f / 20.0f, b2 = -0.5f, b4 = 0.25f, b5 = -1.0f / 12.0f;
    const float h2 = __fmul_rn(h, h), u2 = __fmul_rn(u, u);
    w[0] = __fmul_rn(__fmul_rn(__fmul_rn(u2, u2), u), c120);
    w[5] = __fmul_rn(__fmul_rn(__fmul_rn(h2, h2), h), c120);
    w[1] = __fmaf_rn(h, __fmaf_rn(h, __fmaf_rn(h, __fmaf_rn(h, __fmaf_rn(h, a5, a4), a3), a2), a1), a0);
    w[4] = __fmaf_rn(u, __fmaf_rn(u, __fmaf_rn(u, __fmaf_rn(u, __fmaf_rn(u, a5, a4), a3), a2), a1), a0);
    w[2] = __fmaf_rn(h2, __fmaf_rn(h2, __fmaf_rn(h, b5, b4), b2), b0);
    w[3] = __fmaf_rn(u2, __fmaf_rn(u2, __fmaf_rn(u, b5, b4), b2), b0);
  }
}

// Stencil bases and offsets of one particle for the two staggerings
// (src/Particle.mm:83-94): node-centred (floor(x)) and half-shifted
// (floor(x - 1/2)).
struct Stagger {
  int node, half;
  float hnode, hhalf;
};
__device__ __forceinline__ Stagger stagger(int i, float o) {
  Stagger s;
  s.node = i;
  s.hnode = o;
  if (o >= 0.5f) {
    s.half = i;
    s.hhalf = __fsub_rn(o, 0.5f);
  } else {
    s.half = i - 1;
    s.hhalf = __fadd_rn(o, 0.5f);
  }
  return s;
}

__device__ __forceinline__ long long quant40(float w) { return __float2ll_rn(__fmul_rn(w, kQuant)); }

__device__ __forceinline__ void red_add(float* p, float v) { atomicAdd(p, v); }
__device__ __forceinline__ void red_add(long long* p, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(v));
}

}  // namespace kern
}  // namespace gample
