// common.cuh -- shared helpers of liblaph_gpu.so: status plumbing, complex
// arithmetic in FP64/FP32, lattice index arithmetic.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

#include "../../include/laph_gpu.h"
#include "check.cuh"

namespace laph {

// Per-thread last error message (laph_last_error()).
void set_error(const char* fmt, ...);

#define LAPH_CUDA_TRY(expr)                                                                  \
  do {                                                                                       \
    cudaError_t _e = (expr);                                                                 \
    if (_e != cudaSuccess) {                                                                 \
      ::laph::set_error("%s:%d: %s: %s", __FILE__, __LINE__, #expr, cudaGetErrorString(_e)); \
      return LAPH_ECUDA;                                                                     \
    }                                                                                        \
  } while (0)

#define LAPH_TRY(expr)            \
  do {                            \
    int _s = (expr);              \
    if (_s != LAPH_OK) return _s; \
  } while (0)

// ---------------------------------------------------------------- complex ---
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
__host__ __device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cscal(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
// acc += a*b
__host__ __device__ __forceinline__ void cfma(double2& acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
// acc += conj(a)*b
__host__ __device__ __forceinline__ void cfmac(double2& acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
}
__host__ __device__ __forceinline__ void cfmaf(float2& acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(-a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y);
  acc.y = fmaf(a.y, b.x, acc.y);
}
__host__ __device__ __forceinline__ void cfmacf(float2& acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y);
  acc.y = fmaf(-a.y, b.x, acc.y);
}

// ------------------------------------------------------------- cp.async ---
// 16-byte global -> shared copy that bypasses L1; ok == false writes zeros and
// reads nothing (src-size 0), src must still be a mapped address.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool ok) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(ok ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// ------------------------------------------------------------ lattice idx ---
// site = x*L*L + y*L + z, periodic (modules/navigation.cpp:27-88).
struct Lat {
  int L, L2, V3;
};
__host__ __device__ __forceinline__ int nb_up(const Lat& g, int x, int y, int z, int dir) {
  if (dir == 0) x = (x + 1 == g.L) ? 0 : x + 1;
  else if (dir == 1) y = (y + 1 == g.L) ? 0 : y + 1;
  else z = (z + 1 == g.L) ? 0 : z + 1;
  return LAPH_IX(x * g.L2 + y * g.L + z, g.V3);
}
__host__ __device__ __forceinline__ int nb_dn(const Lat& g, int x, int y, int z, int dir) {
  if (dir == 0) x = (x == 0) ? g.L - 1 : x - 1;
  else if (dir == 1) y = (y == 0) ? g.L - 1 : y - 1;
  else z = (z == 0) ? g.L - 1 : z - 1;
  return LAPH_IX(x * g.L2 + y * g.L + z, g.V3);
}
__host__ __device__ __forceinline__ void site_xyz(const Lat& g, int s, int& x, int& y, int& z) {
  s = LAPH_IX(s, g.V3);
  x = s / g.L2;
  const int r = s - x * g.L2;
  y = r / g.L;
  z = r - y * g.L;
}
__host__ __device__ __forceinline__ int site_up(const Lat& g, int s, int dir) {
  int x, y, z;
  site_xyz(g, s, x, y, z);
  return nb_up(g, x, y, z, dir);
}
__host__ __device__ __forceinline__ int site_dn(const Lat& g, int s, int dir) {
  int x, y, z;
  site_xyz(g, s, x, y, z);
  return nb_dn(g, x, y, z, dir);
}

inline Lat make_lat(int L) { return Lat{L, L * L, L * L * L}; }

inline unsigned ceil_div(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

// [a, a + bytes) and [b, b + bytes) share a byte
inline bool ranges_overlap(const void* a, const void* b, size_t bytes) {
  const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
  return x < y + bytes && y < x + bytes;
}

}  // namespace laph
