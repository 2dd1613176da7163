// filter_variants.cuh -- the filter variants 2-5 (filter_variants.cu): the same
// step as the default kernel with its operands or links held elsewhere (tensor
// memory, a bulk-copy pipeline, 512-site bricks, a per-thread cp.async buffer);
// each gives the default's results bit for bit and measured slower.
#pragma once
#include "batch.cuh"

namespace laph {
// Opt the variants into their dynamic shared memory on the current device.
int cheb_variants_init();
// One filter step with variant 2-5 (the arguments of cheb_step).
int cheb_variant_step(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, int kb, int bf16,
                      const void* links, const float* scale, const float2* X, const float2* Z, const float2* S,
                      float2* Y, const double2* V, double2* W, const double* tcoef, int step, bool final_step,
                      int variant, int tile, int lmax, int* err, cudaStream_t st);
}  // namespace laph
