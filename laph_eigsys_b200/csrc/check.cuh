// check.cuh -- index checks of the bounds-checked build (-DLAPH_CHECK,
// liblaph_gpu_check.so).
//
// LAPH_IX(i, n) is the index i, checked against [0, n) in the checked build.
// An index outside the range is counted and the first one recorded (value,
// bound, source line, translation unit), and the access it was meant for goes
// to index 0 instead, so a checked kernel records the fault and never makes
// it: nothing traps, nothing reads or writes out of bounds.  Each translation
// unit that includes this header keeps its own record in device memory and
// registers a reader for it with the library at load time;
// laph_check_report() sums the records of all translation units.  In the
// normal build LAPH_IX(i, n) is i and nothing else is compiled.
#pragma once
#include <cuda_runtime.h>

namespace laph {

struct CheckRec {
  unsigned long long count;  // indices found out of range
  long long index, bound;    // the first one and its bound
  int line;                  // source line of the first one's LAPH_IX
  int pad;
};
using CheckReader = int (*)(CheckRec* out, int reset, const char** unit);
void check_register(CheckReader fn);

#ifdef LAPH_CHECK
namespace {
__device__ CheckRec g_check_rec;

int check_read_unit(CheckRec* out, int reset, const char** unit) {
  if (unit) *unit = __BASE_FILE__;
  if (cudaMemcpyFromSymbol(out, g_check_rec, sizeof(CheckRec)) != cudaSuccess) return 1;
  if (reset) {
    const CheckRec zero{};
    if (cudaMemcpyToSymbol(g_check_rec, &zero, sizeof(CheckRec)) != cudaSuccess) return 1;
  }
  return 0;
}
struct CheckUnitRegistration {
  CheckUnitRegistration() { check_register(&check_read_unit); }
};
const CheckUnitRegistration g_check_unit_registration;
}  // namespace

template <typename T>
__device__ __forceinline__ T check_ix(T i, long long n, int line) {
  const long long v = (long long)i;
  if (v >= 0 && v < n) return i;
  if (atomicAdd(&g_check_rec.count, 1ull) == 0ull) {
    g_check_rec.index = v;
    g_check_rec.bound = n;
    g_check_rec.line = line;
  }
  return T(0);
}
#ifdef __CUDA_ARCH__
#define LAPH_IX(i, n) ::laph::check_ix((i), (long long)(n), __LINE__)
#else
#define LAPH_IX(i, n) (i)
#endif
#else
#define LAPH_IX(i, n) (i)
#endif

}  // namespace laph
