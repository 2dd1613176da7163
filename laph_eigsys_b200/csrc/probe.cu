// probe.cu -- laph_probe_fp64: the device's FP64 peaks measured in place, as
// the denominators of the FP64 kernels' rooflines (the Gram, the rotation, the
// source-shape tile), so that a report quotes a peak measured on the same part
// at the same moment instead of a constant.  Two saturating loops, each timed
// with CUDA events over a few launches on a private stream:
//   FMA : every thread runs 8 independent chains of dependent fma.rn.f64;
//   DMMA: every warp runs 8 independent chains of mma.sync.m8n8k4.f64
//         (512 flop each), the FP64 tensor path the dense kernels use.
// Grid: 8 CTAs of 256 threads per SM.  The results feed a sum written to
// device memory, so the loops cannot be removed.
#include "common.cuh"

namespace laph {
namespace {

constexpr int kProbeIters = 4096;
constexpr int kChains = 8;

__global__ void __launch_bounds__(256) k_probe_fma(double* out, double seed) {
  double a[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) a[c] = seed + threadIdx.x * 1e-9 + c;
  const double m = 1.0 + 1e-12, b = 1e-13;
#pragma unroll 4
  for (int i = 0; i < kProbeIters; ++i)
#pragma unroll
    for (int c = 0; c < kChains; ++c) a[c] = fma(a[c], m, b);
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += a[c];
  if (s == 12345.678) out[blockIdx.x] = s;  // never true; keeps the chains live
}

__global__ void __launch_bounds__(256) k_probe_dmma(double* out, double seed) {
  double acc[kChains][2];
#pragma unroll
  for (int c = 0; c < kChains; ++c) acc[c][0] = acc[c][1] = 0.0;
  const double a = seed + threadIdx.x * 1e-9, b = 1e-3;
#pragma unroll 4
  for (int i = 0; i < kProbeIters; ++i)
#pragma unroll
    for (int c = 0; c < kChains; ++c)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                   : "+d"(acc[c][0]), "+d"(acc[c][1])
                   : "d"(a), "d"(b));
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += acc[c][0] + acc[c][1];
  if (s == 12345.678) out[blockIdx.x] = s;
}

}  // namespace
}  // namespace laph

using namespace laph;

extern "C" int laph_probe_fp64(int device, double* fma_tflops, double* dmma_tflops) {
  if (!fma_tflops || !dmma_tflops) {
    set_error("laph_probe_fp64: null pointer");
    return LAPH_EINVAL;
  }
  LAPH_CUDA_TRY(cudaSetDevice(device));
  int sms = 0;
  LAPH_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  const int grid = 8 * sms, reps = 5;
  cudaStream_t st;
  LAPH_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  double* out = nullptr;
  cudaEvent_t e0, e1;
  int rc = LAPH_OK;
  if (cudaMalloc(&out, sizeof(double) * grid) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
      cudaEventCreate(&e1) != cudaSuccess) {
    cudaGetLastError();
    cudaStreamDestroy(st);
    set_error("laph_probe_fp64: set-up failed");
    return LAPH_ECUDA;
  }
  float ms[2] = {0.f, 0.f};
  for (int k = 0; k < 2 && rc == LAPH_OK; ++k) {
    auto launch = [&] {
      if (k == 0) k_probe_fma<<<grid, 256, 0, st>>>(out, 1.0);
      else k_probe_dmma<<<grid, 256, 0, st>>>(out, 1.0);
    };
    launch();  // warm-up
    cudaEventRecord(e0, st);
    for (int r = 0; r < reps; ++r) launch();
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms[k], e0, e1) != cudaSuccess) {
      cudaGetLastError();
      set_error("laph_probe_fp64: probe launch failed");
      rc = LAPH_ECUDA;
    }
  }
  const double threads = (double)grid * 256.0;
  const double fma_flop = threads * kProbeIters * kChains * 2.0 * reps;
  const double dmma_flop = threads / 32.0 * kProbeIters * kChains * 512.0 * reps;
  *fma_tflops = ms[0] > 0.f ? fma_flop / (ms[0] * 1e-3) / 1e12 : 0.0;
  *dmma_tflops = ms[1] > 0.f ? dmma_flop / (ms[1] * 1e-3) / 1e12 : 0.0;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  cudaStreamDestroy(st);
  return rc;
}
