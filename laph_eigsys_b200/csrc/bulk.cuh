// bulk.cuh -- shared-memory transaction barriers (mbarrier) and the untiled
// bulk copy engine (cp.async.bulk, global -> this CTA's shared memory).
//
// A stage of a copy pipeline is one mbarrier initialised with one arrival:
// the issuing thread arrives with the stage's byte count (expect_tx), the
// copies complete the transaction, and the phase flips when both are done;
// consumers wait on the phase parity of the stage's n-th use (n & 1).  Every
// copy starts at a 16-byte aligned global address, lands at a 16-byte aligned
// shared address and moves a multiple of 16 bytes.  No copy is multicast.
#pragma once
#include <cstdint>

namespace laph {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* m, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(m)), "r"(count) : "memory");
}
// makes the initialised barriers visible to the copy engine (before the CTA barrier that publishes them)
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* m, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(m)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* m) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(m)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* m, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(m)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Wait for phase `parity` of m, giving up after `limit_ns` nanoseconds of the
// global timer (each try_wait poll suspends the thread for at most a
// hardware-chosen time); returns false on giving up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* m, unsigned parity, unsigned long long limit_ns) {
  if (mbar_try_wait(m, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(m, parity))
    if (global_ns() - t0 > limit_ns) return false;
  return true;
}
// global -> this CTA's shared memory, completing `bytes` on m
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* m) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(m))
               : "memory");
}

}  // namespace laph
