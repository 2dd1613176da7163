// tmem.cuh -- tensor memory (TMEM) as per-thread storage beside the register file.
//
// Each SM has 128 lanes x 512 columns of 32-bit TMEM, allocated per CTA in
// power-of-two column counts (32..512) by one warp.  With the 32x32b access
// shape warp w of a CTA reads and writes lanes 32*(w % 4) .. 32*(w % 4) + 31,
// one lane per thread, so a thread can keep a private row of up to `ncols`
// 32-bit values there and load them back with tcgen05.ld.  The loads go
// through TMEM's own data path, not through L1 / shared memory.
//
// Rules every user of these helpers keeps: the allocating warp is converged
// and allocates once; every CTA that allocated reaches tmem_dealloc on every
// path (no early return after the allocation); the columns a kernel allocates
// per CTA times its resident CTAs per SM stay within 512 (a CTA whose
// allocation does not fit waits until a resident CTA of the same launch frees
// its columns); the destination registers of a tcgen05.ld are read only after
// tmem_wait_ld, which takes them as operands so the compiler keeps that order.
#pragma once
#include <cstdint>

namespace laph {

// one full warp; writes the TMEM base address to *dst (shared memory)
__device__ __forceinline__ void tmem_alloc_warp(uint32_t* dst, uint32_t ncols) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(a), "r"(ncols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
// one full warp of the allocating CTA, after every TMEM access of the CTA ended
__device__ __forceinline__ void tmem_dealloc_warp(uint32_t base, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(base), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tmem_fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
// address of this thread's lane (32x32b shape): lane field = 32 * (warp % 4)
__device__ __forceinline__ uint32_t tmem_lane_addr(uint32_t base, uint32_t col) {
  const uint32_t warp = threadIdx.x >> 5;
  return base + ((32u * (warp & 3u)) << 16) + col;
}

// ---- stores (registers -> this thread's lane, consecutive columns) --------
__device__ __forceinline__ void tmem_st16(uint32_t t, const uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16};\n" ::"r"(t),
      "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
      "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
      : "memory");
}
__device__ __forceinline__ void tmem_st2(uint32_t t, uint32_t a, uint32_t b) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};\n" ::"r"(t), "r"(a), "r"(b) : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory"); }

// ---- loads (this thread's lane -> registers) -------------------------------
__device__ __forceinline__ void tmem_ld16(uint32_t t, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(t));
}
__device__ __forceinline__ void tmem_ld2(uint32_t t, uint32_t& a, uint32_t& b) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];\n" : "=r"(a), "=r"(b) : "r"(t));
}
// waits for this thread's outstanding tcgen05.ld; the 18 registers they
// wrote pass through as operands, so no read of them moves above the wait
__device__ __forceinline__ void tmem_wait_ld18(uint32_t (&v)[16], uint32_t& a, uint32_t& b) {
  asm volatile("tcgen05.wait::ld.sync.aligned;\n"
               : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]), "+r"(v[7]),
                 "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]), "+r"(v[12]), "+r"(v[13]), "+r"(v[14]),
                 "+r"(v[15]), "+r"(a), "+r"(b)
               :
               : "memory");
}

}  // namespace laph
