// stencil64cols.cuh -- the FP64 block stencil (-Delta) of the Rayleigh-Ritz
// step, laid out like the FP32 filter: one thread per site walks a block of
// kColsFP64 columns, the site's 3 forward links in 108 registers and its 3
// backward links U_mu(s - mu) in shared memory (55 KB per CTA, each thread
// reading only its own column, so no barrier), read once per column block
// instead of once per (site, column); colour-major columns, so every warp
// access is a dense 512-byte segment.
#pragma once
#include "batch.cuh"

namespace laph {

constexpr int kColsFP64 = 32;  // columns per CTA
constexpr int kSites64 = 128;  // sites per CTA (threads)

constexpr int kStencil64Smem = 27 * kSites64 * (int)sizeof(double2);  // 55 KB: dynamic, opted in

struct Links64 {
  double2 uf[3][9];
};

// Forward links of site s into registers, backward links into sUb[e][threadIdx.x].
__device__ __forceinline__ void load_links64(const double2* __restrict__ U, const Lat& g, int s, const int* dn,
                                             Links64& l, double2 (*sUb)[kSites64]) {
#pragma unroll
  for (int mu = 0; mu < 3; ++mu)
#pragma unroll
    for (int e = 0; e < 9; ++e) {
      l.uf[mu][e] = __ldg(U + (size_t)(mu * 9 + e) * g.V3 + s);
      sUb[mu * 9 + e][threadIdx.x] = __ldg(U + (size_t)(mu * 9 + e) * g.V3 + dn[mu]);
    }
}

// hop(x)(s) = sum_mu U_mu(s) x(s+mu) + U_mu(s-mu)^dag x(s-mu) on a colour-major column.
__device__ __forceinline__ void hop64_col(const Links64& l, const double2 (*sUb)[kSites64], int V3, const int* up,
                                          const int* dn, const double2* __restrict__ x, double2 acc[3]) {
  acc[0] = acc[1] = acc[2] = make_double2(0.0, 0.0);
#pragma unroll
  for (int mu = 0; mu < 3; ++mu) {
    double2 xu[3], xd[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      xu[b] = __ldg(x + (size_t)b * V3 + up[mu]);
      xd[b] = __ldg(x + (size_t)b * V3 + dn[mu]);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        cfma(acc[a], l.uf[mu][3 * a + b], xu[b]);
        cfmac(acc[a], sUb[mu * 9 + 3 * b + a][threadIdx.x], xd[b]);
      }
  }
}

}  // namespace laph
