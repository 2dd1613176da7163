// filter_common.cuh -- device helpers shared by the filter kernels (filter.cu)
// and their measured alternatives (filter_variants.cu): link loads (FP32, or
// BF16 with a per-site scale), packed FP32x2 arithmetic, the L2 bulk prefetch.
#pragma once
#include <cuda_bf16.h>

#include "batch.cuh"

namespace laph {

// ---------------------------------------------------------------- links ----
__device__ __forceinline__ float2 ld_lk(const float2* __restrict__ p, const float*, size_t i, int) { return __ldg(p + i); }
__device__ __forceinline__ float2 ld_lk(const __nv_bfloat162* __restrict__ p, const float* __restrict__ sc, size_t i,
                                        int site) {
  const float2 v = __bfloat1622float2(__ldg(p + i));
  const float s = __ldg(sc + site);
  return make_float2(v.x * s, v.y * s);
}

// ------------------------------------------------------- packed FP32x2 ----
__device__ __forceinline__ unsigned long long pk2(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ float2 unpk2(unsigned long long v) {
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
  return r;
}
// d += a * b elementwise on (lo, hi) FP32 pairs (sm_100a)
__device__ __forceinline__ void ffma2(unsigned long long& d, unsigned long long a, unsigned long long b) {
  asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(d) : "l"(a), "l"(b));
}

// ------------------------------------------------------ L2 bulk prefetch ---
// columns of lookahead of the L2 bulk prefetch
#ifndef LAPH_PREFETCH_COLS
#define LAPH_PREFETCH_COLS 4
#endif
constexpr int kPrefetch = LAPH_PREFETCH_COLS;
// Bulk prefetch of [p, p+bytes) into L2 (16-byte aligned, bytes % 16 == 0).
__device__ __forceinline__ void l2_prefetch(const void* p, unsigned bytes) {
  if ((reinterpret_cast<uintptr_t>(p) & 15u) == 0 && (bytes & 15u) == 0 && bytes > 0)
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(p), "r"(bytes) : "memory");
}

// column blocks up to this width stage their step coefficients per CTA (variants 1-5)
constexpr int kCoefMax = 64;

}  // namespace laph
