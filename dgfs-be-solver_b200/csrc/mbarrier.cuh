// mbarrier helpers with bounded waits, shared by the cluster-exchange
// collision kernels and the tensor-core GEMM.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace dgfs {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Default limit of one bounded wait: 1 s of %globaltimer.
constexpr uint64_t kWaitLimitNs = 1000000000ull;

// Wait for phase `parity` of `bar`, giving up after `limit_ns`: the wait
// that gives up sets the global flag `err` (read by the host) and the CTA's
// shared flag `gave_up`; every later wait of that CTA returns at once, so a
// failed exchange costs one timeout per CTA, not one per (p, q).  The global
// flag is only written here, never read: a flag left set by an earlier
// launch does not change how this launch waits.
__device__ __forceinline__ void mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err, int* gave_up,
                                                  uint64_t limit_ns = kWaitLimitNs) {
  if (mbar_try_wait(bar, parity)) return;
  const uint64_t t0 = globaltimer_ns();
  for (uint32_t i = 1;; ++i) {
    if (mbar_try_wait(bar, parity)) return;
    if ((i & 255u) == 0) {
      if (*(volatile int*)gave_up) return;
      if (globaltimer_ns() - t0 > limit_ns) {
        atomicExch(err, 1);
        *(volatile int*)gave_up = 1;
        return;
      }
    }
  }
}

}  // namespace dgfs
