// Bulk asynchronous copies (TMA, cp.async.bulk) global -> shared with mbarrier
// completion, for sm_90+ / sm_100a.  Only plain (non-multicast) copies of this
// GPU's own memory are used.  Every wait is bounded.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pbgpu {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Make barrier initialisation visible to the async proxy before first use.
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ uint64_t l2_evict_first_policy() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}

// dst and src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar, uint64_t pol) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Wait for the barrier's phase for at most about limit_ns of wall time (and
// kWaitLimit polls as a backstop; each try_wait may suspend the thread for a
// short hardware-defined time).  Returns false when the limit was reached; a
// zero limit gives up at once without polling (tests drive the timeout path
// with it).
constexpr uint32_t kWaitLimit = 1u << 24;
constexpr uint64_t kWaitNs = 1000000000ull;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase, uint64_t limit_ns = kWaitNs) {
  if (limit_ns == 0) return false;
  if (mbar_try_wait(bar, phase)) return true;
  const uint64_t t0 = global_ns();
  for (uint32_t it = 0; it < kWaitLimit; ++it) {
    if (mbar_try_wait(bar, phase)) return true;
    if ((it & 63u) == 63u && global_ns() - t0 > limit_ns) return false;
  }
  return false;
}

}  // namespace pbgpu
