// cgfd_tma.cuh -- TMA (cp.async.bulk.tensor) and mbarrier helpers for sm_100a.
//
// Every wait is bounded: after kWaitLimit polls the waiting thread records a pipeline
// timeout in the problem's error word and carries on, so a lost transfer ends the kernel
// with an error status instead of a hang.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace cgfd {

constexpr int kWaitLimit = 1 << 22;
constexpr int kErrPipelineTimeout = 2;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Orders this thread's earlier generic-proxy accesses to shared memory before later
// async-proxy (TMA) accesses. A block barrier alone does not: a shared-memory load whose value
// is not yet consumed can still be outstanding when the barrier completes, and a TMA load
// issued after the barrier into the same buffer may then overwrite the data before it is read.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// Bounded wait on phase `parity`; returns false (and flags *err) after `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err, int limit = kWaitLimit) {
  const uint32_t a = smem_u32(bar);
  for (int n = 0; n < limit; ++n) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, P;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  if (err) atomicOr(err, kErrPipelineTimeout);
  return false;
}

// 4-D tiled TMA load (x, y, z, field) into shared memory, completion on `bar`.
// x * 4 bytes must be a multiple of 16 (x a multiple of 4 for float data).
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int x, int y, int z, int f,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(f), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace cgfd
