// Device-side structures and helpers shared by the kernels of the renderer.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device_types.h"
#include "gsr_host.h"

namespace gsr {
// Bound on look-back spins: predecessors always run ahead (tiles are taken
// from an atomic ticket in launch order), so this only guards against a
// fault; on expiry the kernel records kErrLookbackTimeout and moves on.
constexpr uint32_t kSpinLimit = 1u << 22;

__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u32(uint32_t *p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long *p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Single-value decoupled look-back (one warp). Status words hold a 2-bit
// flag (1 = aggregate, 2 = inclusive prefix) in the top bits and the value in
// the low 62 bits. Returns the exclusive prefix of `block`.
constexpr unsigned long long kFlagAgg = 1ull << 62;
constexpr unsigned long long kFlagInc = 2ull << 62;
constexpr unsigned long long kValueMask = (1ull << 62) - 1;

__device__ __forceinline__ unsigned long long lookback_warp(unsigned long long *status,
                                                            uint32_t block,
                                                            unsigned long long aggregate,
                                                            uint32_t *error) {
  const uint32_t lane = threadIdx.x & 31;
  if (block == 0) {
    if (lane == 0) st_relaxed_u64(&status[0], kFlagInc | aggregate);
    return 0;
  }
  if (lane == 0) st_relaxed_u64(&status[block], kFlagAgg | aggregate);
  unsigned long long exclusive = 0;
  int64_t base = (int64_t)block - 1;
  uint32_t spins = 0;
  while (true) {
    int64_t idx = base - (int64_t)lane;
    unsigned long long s = idx >= 0 ? ld_relaxed_u64(&status[idx]) : kFlagInc;
    if (__any_sync(0xffffffffu, (s >> 62) == 0)) {
      if (++spins > kSpinLimit) {
        if (lane == 0) atomicOr(error, kErrLookbackTimeout);
        break;
      }
      __nanosleep(32);
      continue;
    }
    uint32_t inc = __ballot_sync(0xffffffffu, (s >> 62) == 2);
    if (inc) {
      uint32_t first = __ffs(inc) - 1;
      exclusive += warp_sum<unsigned long long>(lane <= first ? (s & kValueMask) : 0ull);
      break;
    }
    exclusive += warp_sum<unsigned long long>(s & kValueMask);
    base -= 32;
  }
  if (lane == 0) st_relaxed_u64(&status[block], kFlagInc | (exclusive + aggregate));
  return exclusive;
}

// Finds the view a block or a global index belongs to: the last v with
// base(v) <= x, by binary search over the view table.
template <typename F>
__device__ __forceinline__ uint32_t find_view(uint32_t num_views, uint32_t x, F base) {
  uint32_t lo = 0, hi = num_views - 1;
  while (lo < hi) {
    uint32_t mid = (lo + hi + 1) >> 1;
    if (base(mid) <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Split form of the look-back for kernels that learn their block's count
// early but can use the prefix only later: publish the aggregate as soon as
// it is known, resolve the exclusive prefix (any warp, read-only) later, and
// have exactly one warp publish the inclusive prefix afterwards.
__device__ __forceinline__ void lookback_publish_aggregate(unsigned long long *status,
                                                           uint32_t block,
                                                           unsigned long long aggregate) {
  st_relaxed_u64(&status[block], (block == 0 ? kFlagInc : kFlagAgg) | aggregate);
}

__device__ __forceinline__ unsigned long long lookback_resolve(unsigned long long *status,
                                                               uint32_t block, uint32_t *error) {
  const uint32_t lane = threadIdx.x & 31;
  if (block == 0) return 0;
  unsigned long long exclusive = 0;
  int64_t base = (int64_t)block - 1;
  uint32_t spins = 0;
  while (true) {
    int64_t idx = base - (int64_t)lane;
    unsigned long long s = idx >= 0 ? ld_relaxed_u64(&status[idx]) : kFlagInc;
    if (__any_sync(0xffffffffu, (s >> 62) == 0)) {
      if (++spins > kSpinLimit) {
        if (lane == 0) atomicOr(error, kErrLookbackTimeout);
        break;
      }
      __nanosleep(32);
      continue;
    }
    uint32_t inc = __ballot_sync(0xffffffffu, (s >> 62) == 2);
    if (inc) {
      uint32_t first = __ffs(inc) - 1;
      exclusive += warp_sum<unsigned long long>(lane <= first ? (s & kValueMask) : 0ull);
      break;
    }
    exclusive += warp_sum<unsigned long long>(s & kValueMask);
    base -= 32;
  }
  return exclusive;
}

__device__ __forceinline__ void lookback_publish_inclusive(unsigned long long *status,
                                                           uint32_t block,
                                                           unsigned long long inclusive) {
  if (block != 0) st_relaxed_u64(&status[block], kFlagInc | inclusive);
}

// e^x for x in [-4.5, 0]: Cody-Waite reduction to base 2 and the degree-6
// Taylor polynomial of 2^f (coefficients ln(2)^k / k!), explicit fmaf, so the
// result is reproducible bit for bit by a C++ restatement. Relative error
// about 2e-7. n = rint(t) is taken by adding and subtracting 1.5 * 2^23
// (for |t| < 2^22 the sum rounds t to the nearest integer, ties to even,
// exactly as rintf does), and the same sum's bit pattern gives n as an
// integer: full-rate additions instead of the slower conversion units.
constexpr float kRoundMagic = 12582912.0f;  // 1.5 * 2^23
__device__ __forceinline__ float exp_neg(float x) {
  const float t = __fmul_rn(x, 1.44269504088896341f);
  const float big = __fadd_rn(t, kRoundMagic);
  const float n = __fsub_rn(big, kRoundMagic);
  const float f = __fsub_rn(t, n);
  float p = __fmaf_rn(1.54035304e-4f, f, 1.33335581e-3f);
  p = __fmaf_rn(p, f, 9.61812911e-3f);
  p = __fmaf_rn(p, f, 5.55041087e-2f);
  p = __fmaf_rn(p, f, 2.40226507e-1f);
  p = __fmaf_rn(p, f, 6.93147181e-1f);
  p = __fmaf_rn(p, f, 1.0f);
  const int e = __float_as_int(big) - __float_as_int(kRoundMagic);
  return __int_as_float(__float_as_int(p) + e * (1 << 23));
}

// alpha e^(-4.5 r2) for r2 in [0, 1], the FP32 raster's weight: one fma of
// r2 by -4.5 log2(e) onto log2(alpha) and the hardware base-2 exponential
// (ex2.approx, a few ulp; the argument lies in [-8, 0] on covered pixels, so no subnormal is
// involved). The CPU model of this raster evaluates 2^t with a degree-6
// polynomial instead; the two images agree to the last UNORM8 step except
// where a weight sits on the 1/256 threshold or a channel on a rounding
// boundary.
__device__ __forceinline__ float ex2_approx(float x) {
  float w;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(w) : "f"(x));
  return w;
}

__device__ __forceinline__ float blend_weight(float r2, float log2_alpha) {
  return ex2_approx(fmaf(r2, -6.49212768f, log2_alpha));
}

__device__ __forceinline__ uint32_t to_unorm8(float x) {
  return __float2uint_rn(fminf(fmaxf(x, 0.0f), 1.0f) * 255.0f);
}

// ---- bulk copies global -> shared (TMA, into this CTA only) ----------------
// One elected thread arms an mbarrier with the byte count and issues
// cp.async.bulk copies that complete on it; every thread waits on the
// barrier's phase with a bounded spin. Addresses and sizes must be multiples
// of 16 bytes.
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

// Makes barrier initialisation visible to the asynchronous (TMA) proxy.
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Retires a barrier before its shared memory is used for anything else.
__device__ __forceinline__ void mbar_inval(uint64_t *bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes,
                                              uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Waits for phase `parity` of the barrier; false (and the error bit set)
// when the iteration limit expires.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t *error) {
  uint32_t spins = 0;
  while (!mbar_try_wait(bar, parity)) {
    if (++spins > kSpinLimit) {
      atomicOr(error, kErrStageTimeout);
      return false;
    }
  }
  return true;
}

}  // namespace gsr
