// tc_gemm.cu -- BF16 GEMM on the 5th-generation tensor cores (sm_100a):
// C[M x N] = A[M x K] * B[N x K]^T, A and B K-major (row-major with K
// contiguous), FP32 accumulation in tensor memory.
//
// One CTA (128 threads) per 128 x BN tile. Per K step of BK elements the
// threads copy A and B with cp.async into one of NS shared-memory stages in
// the canonical no-swizzle K-major layout (8-row x 16-byte core matrices;
// leading byte offset between the two K halves of an MMA, stride byte offset
// between 8-row groups), NS - 1 steps ahead of the tensor core; one elected
// thread issues BK/16 tcgen05.mma (M=128, N=BN, K=16) into a BN-column TMEM
// accumulator and commits to the stage's mbarrier, which gates the stage's
// next refill. Every mbarrier wait is bounded (on time-out the kernel sets an
// error flag, skips the epilogue and still frees its TMEM). Epilogue: each
// warp reads its 32 TMEM lanes (rows) with tcgen05.ld and applies one of the
// fused epilogues.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <stdexcept>

#include "device.hpp"
#include "learned.hpp"

namespace gample {
namespace nn {

namespace {

constexpr int BM = 128;
constexpr int kThreads = 128;

__device__ __forceinline__ uint32_t su32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// Shared-memory matrix descriptor (sm100 layout: start >> 4 in [0,14),
// leading byte offset >> 4 in [16,30), stride byte offset >> 4 in [32,46),
// version 1 in [46,48), no swizzle).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return uint64_t((saddr >> 4) & 0x3FFF) | (uint64_t((lbo >> 4) & 0x3FFF) << 16) |
         (uint64_t((sbo >> 4) & 0x3FFF) << 32) | (uint64_t(1) << 46);
}

// Instruction descriptor: F32 accumulator, BF16 A and B, both K-major, M=128.
template <int BN>
__host__ __device__ constexpr uint32_t idesc() {
  return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(BN >> 3) << 17) | (uint32_t(BM >> 4) << 24);
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase) {
  const uint32_t addr = su32(bar);
  for (int i = 0; i < (1 << 20); ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

template <int BN, int BK>
__host__ __device__ constexpr int stage_bytes() {
  return (BM + BN) * BK * 2;
}
// Stages in flight: up to 96 KB of shared memory, so that two CTAs share an SM.
template <int BN, int BK>
__host__ __device__ constexpr int stages() {
  return 4 * stage_bytes<BN, BK>() <= 96 * 1024 ? 4 : 3;
}

// 16-byte global -> shared copy; src_bytes 0 fills the destination with zeros
// (the source is not read).
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int BN, int BK>
__global__ void __launch_bounds__(kThreads) k_gemm(const __nv_bfloat16* __restrict__ A,
                                                   const __nv_bfloat16* __restrict__ B, int M, int N, int K,
                                                   GemmEpilogue ep, int* err, ConvA conv) {
  static_assert(BN == 32 || BN == 64 || BN == 128, "BN");
  static_assert(BK == 32 || BK == 64, "BK");
  constexpr int NS = stages<BN, BK>();
  extern __shared__ __align__(128) unsigned char gsm[];
  __shared__ __align__(8) uint64_t mbar[NS];
  __shared__ __align__(8) uint64_t mbar_drain;  // time-out path: completion of every MMA issued
  __shared__ uint32_t tbase;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  // split K over blockIdx.z (chunks of whole BK steps)
  const int ksteps = K / BK, per = (ksteps + gridDim.z - 1) / gridDim.z;
  const int kbeg = blockIdx.z * per * BK, kend = min(K, (int(blockIdx.z) + 1) * per * BK);
  const int nsteps = kend > kbeg ? (kend - kbeg) / BK : 0;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tbase)), "r"(BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int i = 0; i < NS; ++i) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&mbar[i])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&mbar_drain)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tbase;
  const uint32_t base = su32(gsm);
  // Each thread copies the same 16-byte column kc of rows r0 + j * RS of
  // every tile, so the rows' pixel coordinates (implicit im2col) are found
  // once; per K step only the tap and channel offsets change.
  constexpr int KC = BK / 8, RS = kThreads / KC, RA = BM / RS, RB = BN / RS;
  const int kc = tid % KC, r0 = tid / KC;
  int py[RA], px[RA];
#pragma unroll
  for (int j = 0; j < RA; ++j) {
    const int p = m0 + r0 + j * RS;
    py[j] = conv.x ? p / conv.w : 0;
    px[j] = conv.x ? p - py[j] * conv.w : 0;
    if (conv.x && p >= conv.h * conv.w) py[j] = -(1 << 20);  // padding row: zeros
  }
  // copies of K step t (within this CTA's range) into stage t % NS
  auto load_step = [&](int t) {
    const int k0 = kbeg + t * BK;
    const uint32_t sA = base + uint32_t((t % NS) * stage_bytes<BN, BK>());
    const uint32_t sB = sA + BM * BK * 2;
    const uint32_t col = uint32_t(kc * (BM / 8) * 128);
    if (conv.x) {  // implicit im2col: this K step lies in one tap of the 3 x 3 stencil
      const int tap = k0 / conv.cin, c0 = k0 - tap * conv.cin;
      const int dy = tap / 3 - 1, dx = tap % 3 - 1;
      const __nv_bfloat16* xc = conv.x + c0 + kc * 8;
#pragma unroll
      for (int j = 0; j < RA; ++j) {
        const int m = r0 + j * RS, sy = py[j] + dy, sx = px[j] + dx;
        const bool in = sy >= 0 && sy < conv.h && sx >= 0 && sx < conv.w;
        cp_async16(sA + col + uint32_t((m / 8) * 128 + (m % 8) * 16),
                   in ? xc + (size_t(sy) * conv.w + sx) * conv.cin : conv.x, in ? 16 : 0);
      }
    } else {
#pragma unroll
      for (int j = 0; j < RA; ++j) {
        const int m = r0 + j * RS;
        cp_async16(sA + col + uint32_t((m / 8) * 128 + (m % 8) * 16), A + size_t(m0 + m) * K + k0 + kc * 8, 16);
      }
    }
    const uint32_t colb = uint32_t(kc * (BN / 8) * 128);
#pragma unroll
    for (int j = 0; j < RB; ++j) {
      const int n = r0 + j * RS;
      cp_async16(sB + colb + uint32_t((n / 8) * 128 + (n % 8) * 16), B + size_t(n0 + n) * K + k0 + kc * 8, 16);
    }
  };
  uint32_t phase[NS];
#pragma unroll
  for (int i = 0; i < NS; ++i) phase[i] = 0;
  bool ok = true;
  // Copies run NS - 2 steps ahead; step t refills the stage of step t - 2,
  // whose MMAs had a whole step to finish, so the tensor core gets step t's
  // MMAs queued behind step t - 1's. One commit group per step (empty past
  // the end): "all but the newest NS - 2 groups complete" means "step t has
  // landed".
#pragma unroll
  for (int t = 0; t < NS - 2; ++t) {
    if (t < nsteps) load_step(t);
    cp_async_commit();
  }
  for (int t = 0; t < nsteps && ok; ++t) {
    const int tn = t + NS - 2;
    if (tn < nsteps) {
      bool free_stage = true;
      if (t >= 2) {
        const int sp = (t - 2) % NS;
        free_stage = mbar_wait(&mbar[sp], phase[sp]);  // the MMAs of step t - 2 have read it
        phase[sp] ^= 1;
      }
      if (free_stage) load_step(tn);
      ok = ok && free_stage;
    }
    cp_async_commit();
    cp_async_wait<NS - 2>();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    // every thread leaves the loop together when any wait gave up
    ok = __syncthreads_and(ok) != 0;
    if (!ok) break;
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t aaddr = base + uint32_t((t % NS) * stage_bytes<BN, BK>()), baddr = aaddr + BM * BK * 2;
#pragma unroll
      for (int ks = 0; ks < BK / 16; ++ks) {
        const uint64_t da = sdesc(aaddr + ks * 2 * (BM / 8) * 128, (BM / 8) * 128, 128);
        const uint64_t db = sdesc(baddr + ks * 2 * (BN / 8) * 128, (BN / 8) * 128, 128);
        const uint32_t acc = (t > 0 || ks > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(
                tmem),
            "l"(da), "l"(db), "r"(idesc<BN>()), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       su32(&mbar[t % NS]))
                   : "memory");
    }
  }
  cp_async_wait<0>();  // no copy may still be landing when the CTA ends
  // drain: MMAs complete in order; every earlier completion of the last
  // step's barrier has been waited for, so its phase is current
  if (ok && nsteps > 0) {
    const int sl = (nsteps - 1) % NS;
    ok = mbar_wait(&mbar[sl], phase[sl]);
  }
  ok = __syncthreads_and(ok) != 0;
  if (!ok) {
    // A wait gave up: MMAs already issued may still read the stages and write
    // the accumulator. One more commit arrives on mbar_drain once all of them
    // are complete; wait for it (bounded) before the columns are released.
    // The launch reports the error either way, so its output is discarded.
    if (tid == 0)
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       su32(&mbar_drain))
                   : "memory");
    const bool drained = mbar_wait(&mbar_drain, 0);
    if (tid == 0) atomicExch(err, drained ? 1 : 2);
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok && kbeg < kend) {
    const int row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 16) {
      uint32_t r[16];
      tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + uint32_t(c0), r);
      if (row >= ep.m_valid) continue;
      if (gridDim.z == 1 && n0 + c0 + 16 <= ep.n_valid) {  // 16 whole columns: vector stores when aligned
        float v[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          v[j] = __uint_as_float(r[j]) * ep.alpha;
          if (ep.bias) v[j] += ep.bias[n0 + c0 + j];
          if (ep.relu) v[j] = fmaxf(v[j], 0.0f);
        }
        const size_t o = size_t(row) * ep.ldo + n0 + c0;
        bool done = true;
        if (ep.out_f32) {
          float* q = ep.out_f32 + o;
          if ((reinterpret_cast<uintptr_t>(q) & 15) == 0) {
#pragma unroll
            for (int j = 0; j < 16; j += 4) {
              float4 w4 = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
              if (ep.accumulate) {
                const float4 old = *reinterpret_cast<const float4*>(q + j);
                w4.x += old.x;
                w4.y += old.y;
                w4.z += old.z;
                w4.w += old.w;
              }
              *reinterpret_cast<float4*>(q + j) = w4;
            }
          } else {
            done = false;
          }
        }
        if (ep.out_bf16 && done) {
          __nv_bfloat16* q = ep.out_bf16 + o;
          if ((reinterpret_cast<uintptr_t>(q) & 15) == 0) {
            uint32_t w[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              const __nv_bfloat162 h2 = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
              w[j] = *reinterpret_cast<const uint32_t*>(&h2);
            }
            reinterpret_cast<uint4*>(q)[0] = make_uint4(w[0], w[1], w[2], w[3]);
            reinterpret_cast<uint4*>(q)[1] = make_uint4(w[4], w[5], w[6], w[7]);
          } else if (!ep.out_f32) {
            done = false;
          } else {
#pragma unroll
            for (int j = 0; j < 16; ++j) q[j] = __float2bfloat16_rn(v[j]);
          }
        }
        if (done) continue;
      }
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int n = n0 + c0 + j;
        if (n >= ep.n_valid) continue;
        float v = __uint_as_float(r[j]) * ep.alpha;
        if (gridDim.z > 1) {  // split K: partial sums added atomically (output zeroed by the caller)
          atomicAdd(ep.out_f32 + size_t(row) * ep.ldo + n, v);
          continue;
        }
        if (ep.bias) v += ep.bias[n];
        if (ep.relu) v = fmaxf(v, 0.0f);
        if (ep.out_f32) {
          const size_t o = size_t(row) * ep.ldo + n;
          ep.out_f32[o] = ep.accumulate ? ep.out_f32[o] + v : v;
        }
        if (ep.out_bf16) ep.out_bf16[size_t(row) * ep.ldo + n] = __float2bfloat16_rn(v);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN) : "memory");
}

template <int BN, int BK>
void launch_k(dim3 grid, const __nv_bfloat16* A, const __nv_bfloat16* B, int M, int N, int K, const GemmEpilogue& ep,
              int* err, cudaStream_t s, const ConvA& conv) {
  constexpr int bytes = stages<BN, BK>() * stage_bytes<BN, BK>();
  static std::once_flag once;  // per instantiation; shared by concurrent callers
  std::call_once(once, [] {
    GP_CUDA(cudaFuncSetAttribute(k_gemm<BN, BK>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  });
  if (conv.x && (conv.cin % BK != 0 || K != 9 * conv.cin))
    throw std::invalid_argument("gemm_bf16: implicit im2col needs K = 9 cin and cin a multiple of the K step");
  k_gemm<BN, BK><<<grid, kThreads, bytes, s>>>(A, B, M, N, K, ep, err, conv);
}

template <int BN>
void launch_bn(const __nv_bfloat16* A, const __nv_bfloat16* B, int M, int N, int K, const GemmEpilogue& ep, int* err,
               cudaStream_t s, const ConvA& conv) {
  // split K when the output has few tiles and K is long (weight gradients)
  const int tiles = (N / BN) * (M / BM);
  const int ksteps = K / (K % 64 == 0 ? 64 : 32);
  int splits = 1;
  if (ep.split_k && tiles < 296 && ksteps >= 16) {
    splits = std::min(296 / tiles, ksteps / 8);
    if (splits < 1) splits = 1;
  }
  if (splits > 1) {
    if (!ep.out_f32 || ep.bias || ep.relu || ep.out_bf16 || ep.accumulate)
      throw std::invalid_argument("gemm_bf16: split K needs a plain FP32 output");
    if (ep.ldo == ep.n_valid)
      GP_CUDA(cudaMemsetAsync(ep.out_f32, 0, size_t(ep.m_valid) * ep.ldo * sizeof(float), s));
    else
      for (int r = 0; r < ep.m_valid; ++r)
        GP_CUDA(cudaMemsetAsync(ep.out_f32 + size_t(r) * ep.ldo, 0, size_t(ep.n_valid) * sizeof(float), s));
  }
  dim3 grid(N / BN, M / BM, splits);
  if (K % 64 == 0 && (!conv.x || conv.cin % 64 == 0))
    launch_k<BN, 64>(grid, A, B, M, N, K, ep, err, s, conv);
  else
    launch_k<BN, 32>(grid, A, B, M, N, K, ep, err, s, conv);
  GP_LAUNCH_CHECK();
}

}  // namespace

void gemm_bf16(const __nv_bfloat16* A, const __nv_bfloat16* B, int M, int N, int K, const GemmEpilogue& ep, int* err,
               cudaStream_t s, const ConvA& conv) {
  if (M <= 0 || N <= 0 || K <= 0 || M % BM != 0 || K % 32 != 0)
    throw std::invalid_argument("gemm_bf16: M must be a multiple of 128 and K of 32");
  if (N % 128 == 0)
    launch_bn<128>(A, B, M, N, K, ep, err, s, conv);
  else if (N % 64 == 0)
    launch_bn<64>(A, B, M, N, K, ep, err, s, conv);
  else if (N % 32 == 0)
    launch_bn<32>(A, B, M, N, K, ep, err, s, conv);
  else
    throw std::invalid_argument("gemm_bf16: N must be a multiple of 32");
}

}  // namespace nn
}  // namespace gample
