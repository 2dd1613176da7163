// check.cu -- the report of the bounds-checked build (check.cuh): every
// translation unit's record of out-of-range indices, summed; and a self-test
// kernel that shows one being recorded.
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace laph {

static std::vector<CheckReader>& check_readers() {
  static std::vector<CheckReader> r;
  return r;
}
static std::mutex g_check_mu;

void check_register(CheckReader fn) {
  std::lock_guard<std::mutex> lk(g_check_mu);
  check_readers().push_back(fn);
}

#ifdef LAPH_CHECK
// Checks index n + 3 against [0, n): recorded, and the store goes to element 0.
__global__ void k_check_selftest(int* buf, int n) {
  if (threadIdx.x == 0 && blockIdx.x == 0) buf[LAPH_IX(n + 3, n)] = 7;
}
#endif

}  // namespace laph

using namespace laph;

extern "C" int laph_check_enabled(void) {
#ifdef LAPH_CHECK
  return 1;
#else
  return 0;
#endif
}

extern "C" int laph_check_report(unsigned long long* count, long long* index, long long* bound, int* line, char* unit,
                                 int unit_len, int reset) {
  if (!count) {
    set_error("laph_check_report: count is NULL");
    return LAPH_EINVAL;
  }
  *count = 0;
  bool first = true;
  std::lock_guard<std::mutex> lk(g_check_mu);
  for (CheckReader fn : check_readers()) {
    CheckRec r{};
    const char* u = nullptr;
    if (fn(&r, reset, &u) != 0) {
      cudaGetLastError();
      set_error("laph_check_report: cannot read the record of %s", u ? u : "?");
      return LAPH_ECUDA;
    }
    if (r.count == 0) continue;
    *count += r.count;
    if (first) {
      first = false;
      if (index) *index = r.index;
      if (bound) *bound = r.bound;
      if (line) *line = r.line;
      if (unit && unit_len > 0) {
        std::strncpy(unit, u ? u : "", (size_t)unit_len - 1);
        unit[unit_len - 1] = '\0';
      }
    }
  }
  return LAPH_OK;
}

extern "C" int laph_check_selftest(int device) {
#ifdef LAPH_CHECK
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    set_error("laph_check_selftest: cannot use device %d", device);
    return LAPH_ENODEV;
  }
  int* buf = nullptr;
  LAPH_CUDA_TRY(cudaMalloc(&buf, 16 * sizeof(int)));
  k_check_selftest<<<1, 32>>>(buf, 16);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  int v = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&v, buf, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(buf);
  if (e != cudaSuccess) {
    set_error("laph_check_selftest: %s", cudaGetErrorString(e));
    return LAPH_ECUDA;
  }
  if (v != 7) {
    set_error("laph_check_selftest: the checked store did not land at element 0");
    return LAPH_ECUDA;
  }
  return LAPH_OK;
#else
  (void)device;
  set_error("laph_check_selftest: bounds checks are compiled only into liblaph_gpu_check.so (-DLAPH_CHECK)");
  return LAPH_EINVAL;
#endif
}
