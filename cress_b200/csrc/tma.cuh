// TMA (cp.async.bulk.tensor) and mbarrier helpers for sm_100a kernels.
//
// Every wait on an mbarrier is bounded: after kSpinLimit unsuccessful
// try_wait probes the caller gets `false` and must record the failure in
// its error word and leave the kernel (no spin can hang the GPU).
#pragma once
#include <cuda.h>
#include <cstdint>

namespace cress {

constexpr uint32_t kSpinLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Order this thread's earlier generic-proxy shared-memory accesses (made
// visible to it by a preceding __syncthreads) before async-proxy writes.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase with the given parity to complete: at most
// `limit` probes (limit 0 gives up at once, which a test of the failure
// path uses).  A kernel whose wait gave up must stop issuing copies into
// its stages and, before it exits, wait (with the full limit) for every
// copy it issued.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit = kSpinLimit) {
  for (uint32_t n = 0; n < limit; ++n)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// As mbar_try_wait, but the thread may be suspended (taking no issue slots)
// for up to `ns` nanoseconds while the phase is incomplete.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t* bar, uint32_t parity, uint32_t ns) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(ns)
      : "memory");
  return ok != 0;
}

// Bounded wait for a phase expected to take a while (a tensor-core GEMM, a
// producer refilling a stage): at most kSleepProbes probes of up to 1 us
// suspension each, about 2 s in all, so waiting warps leave the issue
// slots to the warps that compute.
constexpr uint32_t kSleepProbes = 1u << 21;
__device__ __forceinline__ bool mbar_wait_sleep(uint64_t* bar, uint32_t parity) {
  for (uint32_t n = 0; n < kSleepProbes; ++n)
    if (mbar_try_wait_sleep(bar, parity, 1000u)) return true;
  return false;
}

// 3-D tiled TMA load of one box into shared memory, completing on `bar`.
// The caller guarantees x*4 bytes is a multiple of 16 (x multiple of 4).
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace cress
