// filter_variants.cu -- measured alternatives of the filter step (filter.cu's
// k_cheb_mrhs2, variant 1), selectable through laph_solve_opts.filter_kernel:
//   2  k_cheb_mrhs3  backward links in tensor memory;
//   3  k_cheb_mrhs4  every vector operand staged by a bulk-copy + mbarrier ring;
//   4  k_cheb_mrhs5  variant 2 on 512-site bricks (one CTA per SM);
//   5  k_cheb_mrhs6  variant 2 with each thread's next-column operands in
//                    flight through cp.async.
// Each runs the default kernel's FMAs in the same order (bitwise the same
// eigenpairs, tested), and each measured slower than the default on the
// 32^3 x 64 workload.
#include "batch.cuh"
#include "bulk.cuh"
#include "filter.cuh"
#include "filter_common.cuh"
#include "filter_variants.cuh"
#include "tmem.cuh"

#include <cuda_bf16.h>

namespace laph {

// Variant 2: k_cheb_mrhs2 with the site's backward links in tensor memory
// instead of shared memory.  In k_cheb_mrhs2 the 27 shared-memory link reads
// per site and column (216 B, two wavefronts per warp read) are about half
// of the L1 / shared-memory data path's work, which is the kernel's busiest
// unit; tcgen05.ld reads them through TMEM's own path.  Each thread keeps its
// 54 link floats in its own TMEM lane: direction mu's first 16 floats at
// columns 16 mu .. 16 mu + 15, its last complex entry at 48 + 2 mu, so one
// direction is one x16 and one x2 load.  A CTA allocates 64 columns (128 for
// the 256-site tile, whose warps 4-7 use columns 64-127 of the same lanes):
// at most 512 per SM at the kernel's residency.  Threads past the end of a
// ragged last tile compute on a clamped site and store nothing, so every warp
// takes part in the warp-wide TMEM instructions.
template <typename LT, bool HAS_Z, bool FINAL, int NT>
__global__ void __launch_bounds__(NT, 512 / NT)
    k_cheb_mrhs3(const ProbDesc* __restrict__ pd, const ProbState* __restrict__ ps, const int* __restrict__ start,
                 int np, int kb, const LT* __restrict__ links, const float* __restrict__ scale,
                 const float2* __restrict__ Xp, const float2* __restrict__ Zp, const float2* __restrict__ Sp,
                 float2* __restrict__ Yp, const double2* __restrict__ Vp, double2* __restrict__ Wp,
                 const double* __restrict__ tcoef, int step) {
  constexpr uint32_t kTmCols = NT > 128 ? 128u : 64u;
  const int p = find_prob(start, np, blockIdx.x);
  if (!ps[p].active) return;
  const ProbDesc d = pd[p];
  const int nst = (d.V3 + NT - 1) / NT;
  const int t = blockIdx.x - start[p];
  const int st = t % nst, cb = t / nst;
  const int s_own = st * NT + threadIdx.x;
  const bool valid = s_own < d.V3;
  const int s = valid ? s_own : d.V3 - 1;
  const int j1 = min(cb * kb + kb, d.k);
  const int nlock = ps[p].nlock;
  if (FINAL && valid) {
    for (int j = cb * kb; j < min(j1, nlock); ++j) {
      const size_t i = (size_t)d.blk + (size_t)j * d.dim + s;
#pragma unroll
      for (int a = 0; a < 3; ++a) Wp[i + (size_t)a * d.V3] = __ldg(Vp + i + (size_t)a * d.V3);
    }
  }
  const int j0 = max(cb * kb, nlock);
  if (j0 >= j1) return;  // uniform over the CTA, before the allocation
  __shared__ float4 cf[kCoefMax];
  __shared__ double ctm[kCoefMax];
  __shared__ uint32_t tm_base;
  {
    const double c_hop = ps[p].c_hop, c_diag = ps[p].c_diag;
    const double* tc = tcoef + d.tc + (size_t)step * 3 * d.k;
    for (int j = j0 + (int)threadIdx.x; j < j1; j += NT) {
      const double a = tc[j];
      cf[LAPH_IX(j - j0, kCoefMax)] = make_float4((float)(a * c_hop), (float)(a * c_diag), (float)tc[d.k + j], (float)tc[2 * d.k + j]);
      if (FINAL) ctm[LAPH_IX(j - j0, kCoefMax)] = tc[(size_t)3 * d.k + j];
    }
  }
  if (threadIdx.x < 32) tmem_alloc_warp(&tm_base, kTmCols);
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  const uint32_t base = tm_base;
  const uint32_t tl = tmem_lane_addr(base, (threadIdx.x >> 7) * 64u);
  const Lat g{d.L, d.L * d.L, d.V3};
  int sx, sy, sz;
  site_xyz(g, s, sx, sy, sz);
  int up[3], dn[3];
#pragma unroll
  for (int mu = 0; mu < 3; ++mu) {
    up[mu] = nb_up(g, sx, sy, sz, mu);
    dn[mu] = nb_dn(g, sx, sy, sz, mu);
  }
  const LT* U = links + d.uf;
  const float* scl = scale + d.sc;
  float2 uf[3][9];
#pragma unroll
  for (int mu = 0; mu < 3; ++mu) {
    uint32_t w[16], w16, w17;
#pragma unroll
    for (int e = 0; e < 9; ++e) {
      uf[mu][e] = ld_lk(U, scl, (size_t)(mu * 9 + e) * d.V3 + s, s);
      const float2 bwl = ld_lk(U, scl, (size_t)(mu * 9 + e) * d.V3 + dn[mu], dn[mu]);
      // stored conjugated for the packed FP32x2 hop
      if (e < 8) {
        w[2 * e] = __float_as_uint(bwl.x);
        w[2 * e + 1] = __float_as_uint(-bwl.y);
      } else {
        w16 = __float_as_uint(bwl.x);
        w17 = __float_as_uint(-bwl.y);
      }
    }
    __syncwarp();
    tmem_st16(tl + 16u * mu, w);
    tmem_st2(tl + 48u + 2u * mu, w16, w17);
  }
  tmem_wait_st();
  const size_t bcol = (size_t)d.blk;
  const int s0 = st * NT, nsite = min(NT, d.V3 - s0);
  const bool pf = threadIdx.x == 0 && (nsite % 2 == 0) && (d.dim % 2 == 0);
  auto prefetch = [&](int j) {
    if (!pf || j >= j1) return;
    const size_t col = bcol + (size_t)j * d.dim;
    const unsigned bytes = 8u * nsite;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      l2_prefetch(Xp + col + (size_t)c * d.V3 + s0, bytes);
      l2_prefetch(Sp + col + (size_t)c * d.V3 + s0, bytes);
      if (HAS_Z) l2_prefetch(Zp + col + (size_t)c * d.V3 + s0, bytes);
    }
    if (FINAL)
#pragma unroll
      for (int c = 0; c < 3; ++c) l2_prefetch(Vp + col + (size_t)c * d.V3 + s0, 2 * bytes);
  };
#pragma unroll 1
  for (int j = j0; j < min(j1, j0 + kPrefetch); ++j) prefetch(j);
#pragma unroll 1
  for (int j = j0; j < j1; ++j) {
    prefetch(j + kPrefetch);
    const size_t col = bcol + (size_t)j * d.dim;
    const float2* x = Xp + col;
    float2 xs[3], ss[3], zz[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      xs[a] = __ldg(x + (size_t)a * d.V3 + s);
      ss[a] = __ldg(Sp + col + (size_t)a * d.V3 + s);
      if (HAS_Z) zz[a] = __ldg(Zp + col + (size_t)a * d.V3 + s);
    }
    unsigned long long P[3] = {0ull, 0ull, 0ull}, T[3] = {0ull, 0ull, 0ull};
#pragma unroll
    for (int mu = 0; mu < 3; ++mu) {
      float2 xu[3], xd[3];
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        xu[b] = __ldg(x + (size_t)b * d.V3 + up[mu]);
        xd[b] = __ldg(x + (size_t)b * d.V3 + dn[mu]);
      }
      uint32_t w[16], w16, w17;
      __syncwarp();  // the TMEM load is warp-wide: reconverge after the prefetch thread and the guarded stores
      tmem_ld16(tl + 16u * mu, w);
      tmem_ld2(tl + 48u + 2u * mu, w16, w17);
      tmem_wait_ld18(w, w16, w17);
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const unsigned long long ur = pk2(xu[b].x, xu[b].x), ui = pk2(xu[b].y, xu[b].y);
        const unsigned long long dr = pk2(xd[b].x, xd[b].x), di = pk2(xd[b].y, xd[b].y);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const int e = 3 * b + a;
          const unsigned long long lf = pk2(uf[mu][3 * a + b].x, uf[mu][3 * a + b].y);
          const unsigned long long lb = e < 8 ? pk2(__uint_as_float(w[2 * e]), __uint_as_float(w[2 * e + 1]))
                                              : pk2(__uint_as_float(w16), __uint_as_float(w17));
          ffma2(P[a], ur, lf);
          ffma2(T[a], ui, lf);
          ffma2(P[a], dr, lb);
          ffma2(T[a], di, lb);
        }
      }
    }
    const float4 q = cf[LAPH_IX(j - j0, kCoefMax)];  // (a c_hop, a c_diag, z, g)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float2 pp = unpk2(P[a]), tt = unpk2(T[a]);
      const float2 acc = make_float2(pp.x - tt.y, pp.y + tt.x);
      float2 r;
      r.x = fmaf(q.x, acc.x, fmaf(q.y, xs[a].x, q.w * ss[a].x));
      r.y = fmaf(q.x, acc.y, fmaf(q.y, xs[a].y, q.w * ss[a].y));
      if (HAS_Z) {
        r.x = fmaf(q.z, zz[a].x, r.x);
        r.y = fmaf(q.z, zz[a].y, r.y);
      }
      if (!valid) continue;
      if (FINAL) {
        const size_t iv = col + (size_t)a * d.V3 + s;
        const double2 v = __ldg(Vp + iv);
        const double tm = ctm[LAPH_IX(j - j0, kCoefMax)];
        Wp[iv] = make_double2(fma(tm, v.x, (double)r.x), fma(tm, v.y, (double)r.y));
      } else {
        Yp[col + (size_t)a * d.V3 + s] = r;
      }
    }
  }
  // every tcgen05.ld of this CTA has been waited for; free the columns
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  if (threadIdx.x < 32) tmem_dealloc_warp(base, kTmCols);
}

// Variant 5: variant 2 with each thread's operands of the next column in
// flight while it computes the current one.  The filter waits on L2: a warp
// issues its 27 loads of a column and then has nothing to do until they
// return.  Here every thread copies its own 27 values of column j + 1 (the 21
// of X at the site and its six neighbours, S, Z) with cp.async into its own
// slots of a two-stage shared-memory buffer, then computes column j from the
// slots filled one column earlier; no thread reads another thread's slots, so
// there is no CTA barrier, only the thread's own cp.async.wait_group.  The
// backward links live in tensor memory (as variant 2), so the buffer (27 x 8 B
// x NT x 2 stages: 55 KB at NT = 128) leaves 4 CTAs per SM.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
constexpr int kPipeSlots = 27;  // per thread and stage: xu[3][3], xd[3][3], xs[3], ss[3], zz[3]

template <typename LT, bool HAS_Z, bool FINAL, int NT>
__global__ void __launch_bounds__(NT, 512 / NT)
    k_cheb_mrhs6(const ProbDesc* __restrict__ pd, const ProbState* __restrict__ ps, const int* __restrict__ start,
                 int np, int kb, const LT* __restrict__ links, const float* __restrict__ scale,
                 const float2* __restrict__ Xp, const float2* __restrict__ Zp, const float2* __restrict__ Sp,
                 float2* __restrict__ Yp, const double2* __restrict__ Vp, double2* __restrict__ Wp,
                 const double* __restrict__ tcoef, int step) {
  constexpr uint32_t kTmCols = NT > 128 ? 128u : 64u;
  const int p = find_prob(start, np, blockIdx.x);
  if (!ps[p].active) return;
  const ProbDesc d = pd[p];
  const int nst = (d.V3 + NT - 1) / NT;
  const int t = blockIdx.x - start[p];
  const int st = t % nst, cb = t / nst;
  const int s_own = st * NT + threadIdx.x;
  const bool valid = s_own < d.V3;
  const int s = valid ? s_own : d.V3 - 1;
  const int j1 = min(cb * kb + kb, d.k);
  const int nlock = ps[p].nlock;
  if (FINAL && valid) {
    for (int j = cb * kb; j < min(j1, nlock); ++j) {
      const size_t i = (size_t)d.blk + (size_t)j * d.dim + s;
#pragma unroll
      for (int a = 0; a < 3; ++a) Wp[i + (size_t)a * d.V3] = __ldg(Vp + i + (size_t)a * d.V3);
    }
  }
  const int j0 = max(cb * kb, nlock);
  if (j0 >= j1) return;  // uniform over the CTA, before the allocation
  __shared__ float4 cf[kCoefMax];
  __shared__ double ctm[kCoefMax];
  __shared__ uint32_t tm_base;
  extern __shared__ __align__(16) float2 pipe[];  // [stage][slot][NT]
  {
    const double c_hop = ps[p].c_hop, c_diag = ps[p].c_diag;
    const double* tc = tcoef + d.tc + (size_t)step * 3 * d.k;
    for (int j = j0 + (int)threadIdx.x; j < j1; j += NT) {
      const double a = tc[j];
      cf[LAPH_IX(j - j0, kCoefMax)] =
          make_float4((float)(a * c_hop), (float)(a * c_diag), (float)tc[d.k + j], (float)tc[2 * d.k + j]);
      if (FINAL) ctm[LAPH_IX(j - j0, kCoefMax)] = tc[(size_t)3 * d.k + j];
    }
  }
  if (threadIdx.x < 32) tmem_alloc_warp(&tm_base, kTmCols);
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  const uint32_t base = tm_base;
  const uint32_t tl = tmem_lane_addr(base, (threadIdx.x >> 7) * 64u);
  const Lat g{d.L, d.L * d.L, d.V3};
  int sx, sy, sz;
  site_xyz(g, s, sx, sy, sz);
  int up[3], dn[3];
#pragma unroll
  for (int mu = 0; mu < 3; ++mu) {
    up[mu] = nb_up(g, sx, sy, sz, mu);
    dn[mu] = nb_dn(g, sx, sy, sz, mu);
  }
  const size_t bcol = (size_t)d.blk;
  // this thread's copies of column j into stage b
  auto issue = [&](int j, int b) {
    float2* sl = pipe + (size_t)b * kPipeSlots * NT + threadIdx.x;
    const size_t col = bcol + (size_t)j * d.dim;
    const float2* x = Xp + col;
#pragma unroll
    for (int mu = 0; mu < 3; ++mu)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        cp_async8(sl + (size_t)(mu * 3 + c) * NT, x + (size_t)c * d.V3 + up[mu]);
        cp_async8(sl + (size_t)(9 + mu * 3 + c) * NT, x + (size_t)c * d.V3 + dn[mu]);
      }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      cp_async8(sl + (size_t)(18 + c) * NT, x + (size_t)c * d.V3 + s);
      cp_async8(sl + (size_t)(21 + c) * NT, Sp + col + (size_t)c * d.V3 + s);
      if (HAS_Z) cp_async8(sl + (size_t)(24 + c) * NT, Zp + col + (size_t)c * d.V3 + s);
    }
  };
  issue(j0, 0);
  cp_async_commit();
  const LT* U = links + d.uf;
  const float* scl = scale + d.sc;
  float2 uf[3][9];
#pragma unroll
  for (int mu = 0; mu < 3; ++mu) {
    uint32_t w[16], w16 = 0, w17 = 0;
#pragma unroll
    for (int e = 0; e < 9; ++e) {
      uf[mu][e] = ld_lk(U, scl, (size_t)(mu * 9 + e) * d.V3 + s, s);
      const float2 bwl = ld_lk(U, scl, (size_t)(mu * 9 + e) * d.V3 + dn[mu], dn[mu]);
      if (e < 8) {
        w[2 * e] = __float_as_uint(bwl.x);
        w[2 * e + 1] = __float_as_uint(-bwl.y);
      } else {
        w16 = __float_as_uint(bwl.x);
        w17 = __float_as_uint(-bwl.y);
      }
    }
    __syncwarp();
    tmem_st16(tl + 16u * mu, w);
    tmem_st2(tl + 48u + 2u * mu, w16, w17);
  }
  tmem_wait_st();
  const int s0 = st * NT, nsite = min(NT, d.V3 - s0);
  const bool pf = threadIdx.x == 0 && (nsite % 2 == 0) && (d.dim % 2 == 0);
  auto prefetch = [&](int j) {
    if (!pf || j >= j1) return;
    const size_t col = bcol + (size_t)j * d.dim;
    const unsigned bytes = 8u * nsite;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      l2_prefetch(Xp + col + (size_t)c * d.V3 + s0, bytes);
      l2_prefetch(Sp + col + (size_t)c * d.V3 + s0, bytes);
      if (HAS_Z) l2_prefetch(Zp + col + (size_t)c * d.V3 + s0, bytes);
    }
    if (FINAL)
#pragma unroll
      for (int c = 0; c < 3; ++c) l2_prefetch(Vp + col + (size_t)c * d.V3 + s0, 2 * bytes);
  };
#pragma unroll 1
  for (int j = j0 + 1; j < min(j1, j0 + 1 + kPrefetch); ++j) prefetch(j);
#pragma unroll 1
  for (int j = j0; j < j1; ++j) {
    const int b = (j - j0) & 1;
    prefetch(j + 1 + kPrefetch);
    if (j + 1 < j1) issue(j + 1, b ^ 1);
    cp_async_commit();  // possibly empty: the group count stays one per column
    cp_async_wait<1>();  // this thread's copies of column j have landed
    const float2* sl = pipe + (size_t)b * kPipeSlots * NT + threadIdx.x;
    const size_t col = bcol + (size_t)j * d.dim;
    unsigned long long P[3] = {0ull, 0ull, 0ull}, T[3] = {0ull, 0ull, 0ull};
#pragma unroll
    for (int mu = 0; mu < 3; ++mu) {
      uint32_t w[16], w16, w17;
      __syncwarp();
      tmem_ld16(tl + 16u * mu, w);
      tmem_ld2(tl + 48u + 2u * mu, w16, w17);
      tmem_wait_ld18(w, w16, w17);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float2 xu = sl[(size_t)(mu * 3 + c) * NT], xd = sl[(size_t)(9 + mu * 3 + c) * NT];
        const unsigned long long ur = pk2(xu.x, xu.x), ui = pk2(xu.y, xu.y);
        const unsigned long long dr = pk2(xd.x, xd.x), di = pk2(xd.y, xd.y);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const int e = 3 * c + a;
          const unsigned long long lf = pk2(uf[mu][3 * a + c].x, uf[mu][3 * a + c].y);
          const unsigned long long lb = e < 8 ? pk2(__uint_as_float(w[2 * e]), __uint_as_float(w[2 * e + 1]))
                                              : pk2(__uint_as_float(w16), __uint_as_float(w17));
          ffma2(P[a], ur, lf);
          ffma2(T[a], ui, lf);
          ffma2(P[a], dr, lb);
          ffma2(T[a], di, lb);
        }
      }
    }
    const float4 q = cf[LAPH_IX(j - j0, kCoefMax)];  // (a c_hop, a c_diag, z, g)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float2 pp = unpk2(P[a]), tt = unpk2(T[a]);
      const float2 acc = make_float2(pp.x - tt.y, pp.y + tt.x);
      const float2 xs = sl[(size_t)(18 + a) * NT], ss = sl[(size_t)(21 + a) * NT];
      float2 rr;
      rr.x = fmaf(q.x, acc.x, fmaf(q.y, xs.x, q.w * ss.x));
      rr.y = fmaf(q.x, acc.y, fmaf(q.y, xs.y, q.w * ss.y));
      if (HAS_Z) {
        const float2 zz = sl[(size_t)(24 + a) * NT];
        rr.x = fmaf(q.z, zz.x, rr.x);
        rr.y = fmaf(q.z, zz.y, rr.y);
      }
      if (!valid) continue;
      if (FINAL) {
        const size_t iv = col + (size_t)a * d.V3 + s;
        const double2 v = __ldg(Vp + iv);
        const double tm = ctm[LAPH_IX(j - j0, kCoefMax)];
        Wp[iv] = make_double2(fma(tm, v.x, (double)rr.x), fma(tm, v.y, (double)rr.y));
      } else {
        Yp[col + (size_t)a * d.V3 + s] = rr;
      }
    }
  }
  cp_async_wait<0>();
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  if (threadIdx.x < 32) tmem_dealloc_warp(base, kTmCols);
}

// Variant 4: variant 2 (backward links in tensor memory) on a 3D tile.  In
// variants 1-3 a CTA owns R whole z-rows of one x-plane, so its x-neighbours
// (one plane away) and the y-rows above and below always come from L2: the
// kernel moves about twice its DRAM bytes from L2 to the SMs.  Here one CTA
// of 512 threads (16 warps, one CTA per SM) owns a TX x 4 x L block (TX =
// 128 / L planes of 4 z-rows each), so most x- and y-neighbours are sites of
// the same CTA, read in the same column at nearly the same time, and hit L1;
// with the links out of shared memory all of the SM's 228 KB serve as L1.
// Each warp is one z-row (L = 32) or part of one, so the loads stay coalesced.
// TMEM: 4 lane groups x 64 columns (warps w, w + 4, w + 8, w + 12 share lanes
// and take columns 64 (w / 4) ..).  Preconditions as variant 3 (host-checked):
// L in {16, 32, 64, 128}.
constexpr int kBrickNT = 512;
constexpr int kBrickTY = 4;

template <typename LT, bool HAS_Z, bool FINAL>
__global__ void __launch_bounds__(kBrickNT, 1)
    k_cheb_mrhs5(const ProbDesc* __restrict__ pd, const ProbState* __restrict__ ps, const int* __restrict__ start,
                 int np, int kb, const LT* __restrict__ links, const float* __restrict__ scale,
                 const float2* __restrict__ Xp, const float2* __restrict__ Zp, const float2* __restrict__ Sp,
                 float2* __restrict__ Yp, const double2* __restrict__ Vp, double2* __restrict__ Wp,
                 const double* __restrict__ tcoef, int step) {
  constexpr uint32_t kTmCols = 256u;
  const int p = find_prob(start, np, blockIdx.x);
  if (!ps[p].active) return;
  const ProbDesc d = pd[p];
  const int L = d.L, L2 = L * L;
  const int TX = kBrickNT / (kBrickTY * L);
  const int nst = d.V3 / kBrickNT;
  const int t = blockIdx.x - start[p];
  const int st = t % nst, cb = t / nst;
  const int nty = L / kBrickTY;
  const int x0 = (st / nty) * TX, y0 = (st % nty) * kBrickTY;
  const int i = threadIdx.x;
  const int zc = i % L, yy = (i / L) % kBrickTY, xx = i / (L * kBrickTY);
  const int s = (x0 + xx) * L2 + (y0 + yy) * L + zc;
  const int j1 = min(cb * kb + kb, d.k);
  const int nlock = ps[p].nlock;
  if (FINAL) {
    for (int j = cb * kb; j < min(j1, nlock); ++j) {
      const size_t ii = (size_t)d.blk + (size_t)j * d.dim + s;
#pragma unroll
      for (int a = 0; a < 3; ++a) Wp[ii + (size_t)a * d.V3] = __ldg(Vp + ii + (size_t)a * d.V3);
    }
  }
  const int j0 = max(cb * kb, nlock);
  if (j0 >= j1) return;  // uniform over the CTA, before the allocation
  __shared__ float4 cf[kCoefMax];
  __shared__ double ctm[kCoefMax];
  __shared__ uint32_t tm_base;
  {
    const double c_hop = ps[p].c_hop, c_diag = ps[p].c_diag;
    const double* tc = tcoef + d.tc + (size_t)step * 3 * d.k;
    for (int j = j0 + i; j < j1; j += kBrickNT) {
      const double a = tc[j];
      cf[LAPH_IX(j - j0, kCoefMax)] = make_float4((float)(a * c_hop), (float)(a * c_diag), (float)tc[d.k + j], (float)tc[2 * d.k + j]);
      if (FINAL) ctm[LAPH_IX(j - j0, kCoefMax)] = tc[(size_t)3 * d.k + j];
    }
  }
  if (i < 32) tmem_alloc_warp(&tm_base, kTmCols);
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  const uint32_t base = tm_base;
  const uint32_t tl = tmem_lane_addr(base, (uint32_t)(i >> 7) * 64u);
  const Lat g{d.L, d.L * d.L, d.V3};
  int sx, sy, sz;
  site_xyz(g, s, sx, sy, sz);
  int up[3], dn[3];
#pragma unroll
  for (int mu = 0; mu < 3; ++mu) {
    up[mu] = nb_up(g, sx, sy, sz, mu);
    dn[mu] = nb_dn(g, sx, sy, sz, mu);
  }
  const LT* U = links + d.uf;
  const float* scl = scale + d.sc;
  float2 uf[3][9];
#pragma unroll
  for (int mu = 0; mu < 3; ++mu) {
    uint32_t w[16], w16 = 0, w17 = 0;
#pragma unroll
    for (int e = 0; e < 9; ++e) {
      uf[mu][e] = ld_lk(U, scl, (size_t)(mu * 9 + e) * d.V3 + s, s);
      const float2 bwl = ld_lk(U, scl, (size_t)(mu * 9 + e) * d.V3 + dn[mu], dn[mu]);
      if (e < 8) {
        w[2 * e] = __float_as_uint(bwl.x);
        w[2 * e + 1] = __float_as_uint(-bwl.y);
      } else {
        w16 = __float_as_uint(bwl.x);
        w17 = __float_as_uint(-bwl.y);
      }
    }
    __syncwarp();
    tmem_st16(tl + 16u * mu, w);
    tmem_st2(tl + 48u + 2u * mu, w16, w17);
  }
  tmem_wait_st();
  // one thread per CTA streams the brick's rows (TX planes x 4 z-rows, contiguous per plane) of the column
  // kPrefetch ahead into L2
  const bool pf = i == 0;
  auto prefetch = [&](int j) {
    if (!pf || j >= j1) return;
    const size_t col = (size_t)d.blk + (size_t)j * d.dim;
    const unsigned bytes = 8u * kBrickTY * L;
    for (int xp = 0; xp < TX; ++xp) {
      const size_t r0 = (size_t)(x0 + xp) * L2 + (size_t)y0 * L;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        l2_prefetch(Xp + col + (size_t)c * d.V3 + r0, bytes);
        l2_prefetch(Sp + col + (size_t)c * d.V3 + r0, bytes);
        if (HAS_Z) l2_prefetch(Zp + col + (size_t)c * d.V3 + r0, bytes);
        if (FINAL) l2_prefetch(Vp + col + (size_t)c * d.V3 + r0, 2 * bytes);
      }
    }
  };
#pragma unroll 1
  for (int j = j0; j < min(j1, j0 + kPrefetch); ++j) prefetch(j);
#pragma unroll 1
  for (int j = j0; j < j1; ++j) {
    prefetch(j + kPrefetch);
    const size_t col = (size_t)d.blk + (size_t)j * d.dim;
    const float2* x = Xp + col;
    unsigned long long P[3] = {0ull, 0ull, 0ull}, T[3] = {0ull, 0ull, 0ull};
#pragma unroll
    for (int mu = 0; mu < 3; ++mu) {
      float2 xu[3], xd[3];
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        xu[b] = __ldg(x + (size_t)b * d.V3 + up[mu]);
        xd[b] = __ldg(x + (size_t)b * d.V3 + dn[mu]);
      }
      uint32_t w[16], w16, w17;
      __syncwarp();
      tmem_ld16(tl + 16u * mu, w);
      tmem_ld2(tl + 48u + 2u * mu, w16, w17);
      tmem_wait_ld18(w, w16, w17);
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const unsigned long long ur = pk2(xu[b].x, xu[b].x), ui = pk2(xu[b].y, xu[b].y);
        const unsigned long long dr = pk2(xd[b].x, xd[b].x), di = pk2(xd[b].y, xd[b].y);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const int e = 3 * b + a;
          const unsigned long long lf = pk2(uf[mu][3 * a + b].x, uf[mu][3 * a + b].y);
          const unsigned long long lb = e < 8 ? pk2(__uint_as_float(w[2 * e]), __uint_as_float(w[2 * e + 1]))
                                              : pk2(__uint_as_float(w16), __uint_as_float(w17));
          ffma2(P[a], ur, lf);
          ffma2(T[a], ui, lf);
          ffma2(P[a], dr, lb);
          ffma2(T[a], di, lb);
        }
      }
    }
    const float4 q = cf[LAPH_IX(j - j0, kCoefMax)];  // (a c_hop, a c_diag, z, g)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float2 pp = unpk2(P[a]), tt = unpk2(T[a]);
      const float2 acc = make_float2(pp.x - tt.y, pp.y + tt.x);
      const size_t ia = col + (size_t)a * d.V3 + s;
      const float2 xs = __ldg(Xp + ia), ss = __ldg(Sp + ia);
      float2 rr;
      rr.x = fmaf(q.x, acc.x, fmaf(q.y, xs.x, q.w * ss.x));
      rr.y = fmaf(q.x, acc.y, fmaf(q.y, xs.y, q.w * ss.y));
      if (HAS_Z) {
        const float2 zz = __ldg(Zp + ia);
        rr.x = fmaf(q.z, zz.x, rr.x);
        rr.y = fmaf(q.z, zz.y, rr.y);
      }
      if (FINAL) {
        const double2 v = __ldg(Vp + ia);
        const double tm = ctm[LAPH_IX(j - j0, kCoefMax)];
        Wp[ia] = make_double2(fma(tm, v.x, (double)rr.x), fma(tm, v.y, (double)rr.y));
      } else {
        Yp[ia] = rr;
      }
    }
  }
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  if (i < 32) tmem_dealloc_warp(base, kTmCols);
}

// Variant 3: the column loop fed by a copy pipeline.  Variants 1 and 2 read
// every vector value with a global load whose latency (an L2 hit, or HBM when
// the bulk prefetch has not landed) the 16 warps of an SM cannot cover: the
// kernel issues at about 55% of the scheduler's rate and waits on loads the
// rest.  Here the CTA's tile is R = NT / L whole z-rows of one x-plane, and
// for each column the first warp, one lane per copy, moves with the bulk copy
// engine into a 3-stage shared-memory ring: the tile's rows of X, its two
// x-neighbour tiles (the same rows one plane up and down, site +- L^2 mod V3),
// the y-neighbour rows above and below the tile (y wraps inside the plane),
// and the tile's rows of S and Z; z-neighbours lie in the tile's own rows.
// Each stage is one mbarrier (one arrival with the stage's byte count);
// the threads wait on it, read every operand from shared memory, and after
// the CTA barrier that ends the column the first warp refills the stage with
// the column kStages ahead.  Backward links stay in tensor memory as in
// variant 2.  Preconditions (host-checked, else the solver uses variant 1):
// L even, NT % L == 0, L^2 % NT == 0, so tiles never straddle planes and
// every copy is 16-byte aligned and a multiple of 16 bytes.  A wait that
// gives up (after kMbarWaitNs) sets *err, waits (bounded) for the copies still
// in flight, frees the tensor memory and ends the CTA.
constexpr int kStages = 3;
constexpr unsigned long long kMbarWaitNs = 1000000000ull;  // 1 s: a stage that takes longer is a fault
constexpr int kStagedNT = 128;    // sites per CTA of the staged variant
constexpr int kStagedMaxL = 128;  // largest lattice extent its ring is sized for
// float2 elements of one stage for lattice extent L, rounded up to 128 bytes:
// X as 3 colours x (tile, x+1 tile, x-1 tile, y+1 row, y-1 row), then S and Z
__host__ __device__ constexpr int stage_stride(int NT, int L) {
  return ((3 * (3 * NT + 2 * L) + 6 * NT) + 15) / 16 * 16;
}

template <typename LT, bool HAS_Z, bool FINAL, int NT>
__global__ void __launch_bounds__(NT, 512 / NT)
    k_cheb_mrhs4(const ProbDesc* __restrict__ pd, const ProbState* __restrict__ ps, const int* __restrict__ start,
                 int np, int kb, const LT* __restrict__ links, const float* __restrict__ scale,
                 const float2* __restrict__ Xp, const float2* __restrict__ Zp, const float2* __restrict__ Sp,
                 float2* __restrict__ Yp, const double2* __restrict__ Vp, double2* __restrict__ Wp,
                 const double* __restrict__ tcoef, int step, int sstride, int* __restrict__ err) {
  constexpr uint32_t kTmCols = NT > 128 ? 128u : 64u;
  const int p = find_prob(start, np, blockIdx.x);
  if (!ps[p].active) return;
  const ProbDesc d = pd[p];
  const int L = d.L, L2 = L * L;
  const int nst = d.V3 / NT;
  const int t = blockIdx.x - start[p];
  const int st = t % nst, cb = t / nst;
  const int s0 = st * NT;
  const int s = s0 + threadIdx.x;
  const int j1 = min(cb * kb + kb, d.k);
  const int nlock = ps[p].nlock;
  if (FINAL) {
    for (int j = cb * kb; j < min(j1, nlock); ++j) {
      const size_t i = (size_t)d.blk + (size_t)j * d.dim + s;
#pragma unroll
      for (int a = 0; a < 3; ++a) Wp[i + (size_t)a * d.V3] = __ldg(Vp + i + (size_t)a * d.V3);
    }
  }
  const int j0 = max(cb * kb, nlock);
  if (j0 >= j1) return;  // uniform over the CTA, before the allocations
  __shared__ float4 cf[kCoefMax];
  __shared__ double ctm[kCoefMax];
  __shared__ uint32_t tm_base;
  __shared__ __align__(8) uint64_t mbar[kStages];
  extern __shared__ __align__(128) float2 stg[];
  {
    const double c_hop = ps[p].c_hop, c_diag = ps[p].c_diag;
    const double* tc = tcoef + d.tc + (size_t)step * 3 * d.k;
    for (int j = j0 + (int)threadIdx.x; j < j1; j += NT) {
      const double a = tc[j];
      cf[LAPH_IX(j - j0, kCoefMax)] = make_float4((float)(a * c_hop), (float)(a * c_diag), (float)tc[d.k + j], (float)tc[2 * d.k + j]);
      if (FINAL) ctm[LAPH_IX(j - j0, kCoefMax)] = tc[(size_t)3 * d.k + j];
    }
  }
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < kStages; ++k) mbar_init(&mbar[k], 1);
    mbar_init_fence();
  }
  if (threadIdx.x < 32) tmem_alloc_warp(&tm_base, kTmCols);
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();

  // tile geometry: R whole z-rows of plane px starting at row y0
  const int R = NT / L;
  const int px = s0 / L2, y0 = (s0 - px * L2) / L;
  const int xu0 = s0 + L2 < d.V3 ? s0 + L2 : s0 + L2 - d.V3;
  const int xd0 = s0 >= L2 ? s0 - L2 : s0 - L2 + d.V3;
  const int yu0 = px * L2 + ((y0 + R) % L) * L;
  const int yd0 = px * L2 + ((y0 + L - 1) % L) * L;
  const int XC = 3 * NT + 2 * L;  // float2 per colour of a stage's X part
  constexpr int kPer = HAS_Z ? 7 : 6;
  const unsigned stage_bytes = 8u * (unsigned)(3 * XC + 3 * NT + (HAS_Z ? 3 * NT : 0));
  // called by all of warp 0: lane l issues copy l of column j into `stage`
  auto issue = [&](int j, int stage) {
    const int lane = threadIdx.x;
    float2* sb = stg + (size_t)stage * sstride;
    const size_t col = (size_t)d.blk + (size_t)j * d.dim;
    const float2* src = nullptr;
    float2* dst = nullptr;
    unsigned n = 0;
    if (lane < 3 * kPer) {
      const int c = lane / kPer, k = lane - c * kPer;
      const size_t cc = col + (size_t)c * d.V3;
      float2* sx = sb + c * XC;
      if (k == 0) { src = Xp + cc + s0; dst = sx; n = NT; }
      else if (k == 1) { src = Xp + cc + xu0; dst = sx + NT; n = NT; }
      else if (k == 2) { src = Xp + cc + xd0; dst = sx + 2 * NT; n = NT; }
      else if (k == 3) { src = Xp + cc + yu0; dst = sx + 3 * NT; n = L; }
      else if (k == 4) { src = Xp + cc + yd0; dst = sx + 3 * NT + L; n = L; }
      else if (k == 5) { src = Sp + cc + s0; dst = sb + 3 * XC + c * NT; n = NT; }
      else { src = Zp + cc + s0; dst = sb + 3 * XC + 3 * NT + c * NT; n = NT; }
    }
    const unsigned bytes = 8u * n;
    const bool ok = n == 0 || ((reinterpret_cast<uintptr_t>(src) & 15u) == 0 &&
                               (reinterpret_cast<uintptr_t>(dst) & 15u) == 0 && (bytes & 15u) == 0);
    const bool all_ok = __all_sync(0xffffffffu, ok);
    if (lane == 0) {
      if (all_ok) {
        mbar_arrive_expect_tx(&mbar[stage], stage_bytes);
      } else {  // never issue a misaligned copy: flag it and complete the phase without data
        atomicExch(err, 2);
        mbar_arrive(&mbar[stage]);
      }
    }
    __syncwarp();
    if (all_ok && n > 0) bulk_g2s(dst, src, bytes, &mbar[stage]);
  };
  if (threadIdx.x < 32)
    for (int it = 0; it < kStages && j0 + it < j1; ++it) issue(j0 + it, it);

  // backward links into this thread's TMEM lane (layout as in variant 2)
  const uint32_t base = tm_base;
  const uint32_t tl = tmem_lane_addr(base, (threadIdx.x >> 7) * 64u);
  const Lat g{d.L, d.L * d.L, d.V3};
  {
    int sx, sy, sz;
    site_xyz(g, s, sx, sy, sz);
    const LT* U = links + d.uf;
    const float* scl = scale + d.sc;
#pragma unroll
    for (int mu = 0; mu < 3; ++mu) {
      const int dnm = nb_dn(g, sx, sy, sz, mu);
      uint32_t w[16], w16 = 0, w17 = 0;
#pragma unroll
      for (int e = 0; e < 9; ++e) {
        const float2 bwl = ld_lk(U, scl, (size_t)(mu * 9 + e) * d.V3 + dnm, dnm);
        if (e < 8) {
          w[2 * e] = __float_as_uint(bwl.x);
          w[2 * e + 1] = __float_as_uint(-bwl.y);
        } else {
          w16 = __float_as_uint(bwl.x);
          w17 = __float_as_uint(-bwl.y);
        }
      }
      __syncwarp();
      tmem_st16(tl + 16u * mu, w);
      tmem_st2(tl + 48u + 2u * mu, w16, w17);
    }
    tmem_wait_st();
  }
  const LT* U = links + d.uf;
  const float* scl = scale + d.sc;
  float2 uf[3][9];
#pragma unroll
  for (int mu = 0; mu < 3; ++mu)
#pragma unroll
    for (int e = 0; e < 9; ++e) uf[mu][e] = ld_lk(U, scl, (size_t)(mu * 9 + e) * d.V3 + s, s);
  // neighbour positions inside a stage's colour block
  const int i = threadIdx.x, r = i / L, zc = i - r * L;
  int upl[3], dnl[3];
  upl[0] = NT + i;
  dnl[0] = 2 * NT + i;
  upl[1] = r < R - 1 ? i + L : 3 * NT + zc;
  dnl[1] = r > 0 ? i - L : 3 * NT + L + zc;
  upl[2] = r * L + (zc + 1 == L ? 0 : zc + 1);
  dnl[2] = r * L + (zc == 0 ? L - 1 : zc - 1);
  const bool pf = FINAL && threadIdx.x == 32;  // V rows into L2 ahead (not staged)
  int jfail = -1;
#pragma unroll 1
  for (int j = j0; j < j1; ++j) {
    const int it = j - j0, stage = it % kStages;
    const unsigned par = (unsigned)(it / kStages) & 1u;
    const size_t col = (size_t)d.blk + (size_t)j * d.dim;
    if (pf && j + kPrefetch < j1) {
      const size_t colp = col + (size_t)kPrefetch * d.dim;
#pragma unroll
      for (int c = 0; c < 3; ++c) l2_prefetch(Vp + colp + (size_t)c * d.V3 + s0, 16u * NT);
    }
    const bool ok = mbar_wait_bounded(&mbar[stage], par, kMbarWaitNs);
    const float2* sb = stg + (size_t)stage * sstride;
    unsigned long long P[3] = {0ull, 0ull, 0ull}, T[3] = {0ull, 0ull, 0ull};
#pragma unroll
    for (int mu = 0; mu < 3; ++mu) {
      float2 xu[3], xd[3];
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        xu[b] = sb[LAPH_IX(b * XC + upl[mu], sstride)];
        xd[b] = sb[LAPH_IX(b * XC + dnl[mu], sstride)];
      }
      uint32_t w[16], w16, w17;
      __syncwarp();
      tmem_ld16(tl + 16u * mu, w);
      tmem_ld2(tl + 48u + 2u * mu, w16, w17);
      tmem_wait_ld18(w, w16, w17);
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const unsigned long long ur = pk2(xu[b].x, xu[b].x), ui = pk2(xu[b].y, xu[b].y);
        const unsigned long long dr = pk2(xd[b].x, xd[b].x), di = pk2(xd[b].y, xd[b].y);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const int e = 3 * b + a;
          const unsigned long long lf = pk2(uf[mu][3 * a + b].x, uf[mu][3 * a + b].y);
          const unsigned long long lb = e < 8 ? pk2(__uint_as_float(w[2 * e]), __uint_as_float(w[2 * e + 1]))
                                              : pk2(__uint_as_float(w16), __uint_as_float(w17));
          ffma2(P[a], ur, lf);
          ffma2(T[a], ui, lf);
          ffma2(P[a], dr, lb);
          ffma2(T[a], di, lb);
        }
      }
    }
    const float4 q = cf[LAPH_IX(j - j0, kCoefMax)];  // (a c_hop, a c_diag, z, g)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float2 pp = unpk2(P[a]), tt = unpk2(T[a]);
      const float2 acc = make_float2(pp.x - tt.y, pp.y + tt.x);
      const float2 xs = sb[LAPH_IX(a * XC + i, sstride)], ss = sb[LAPH_IX(3 * XC + a * NT + i, sstride)];
      float2 rr;
      rr.x = fmaf(q.x, acc.x, fmaf(q.y, xs.x, q.w * ss.x));
      rr.y = fmaf(q.x, acc.y, fmaf(q.y, xs.y, q.w * ss.y));
      if (HAS_Z) {
        const float2 zz = sb[LAPH_IX(3 * XC + 3 * NT + a * NT + i, sstride)];
        rr.x = fmaf(q.z, zz.x, rr.x);
        rr.y = fmaf(q.z, zz.y, rr.y);
      }
      if (FINAL) {
        const size_t iv = col + (size_t)a * d.V3 + s;
        const double2 v = __ldg(Vp + iv);
        const double tm = ctm[LAPH_IX(j - j0, kCoefMax)];
        Wp[iv] = make_double2(fma(tm, v.x, (double)rr.x), fma(tm, v.y, (double)rr.y));
      } else {
        Yp[col + (size_t)a * d.V3 + s] = rr;
      }
    }
    // the stage is free once every thread is past it; a failed wait anywhere ends the loop for the CTA
    if (__syncthreads_or(!ok)) {
      jfail = j;
      break;
    }
    if (threadIdx.x < 32 && j + kStages < j1) issue(j + kStages, stage);
  }
  if (jfail >= 0) {
    if (threadIdx.x == 0) atomicExch(err, 1);
    // columns jfail .. jfail + kStages - 1 may still have copies in flight into this CTA's stages
    for (int j = jfail; j < min(j1, jfail + kStages); ++j) {
      const int it = j - j0;
      mbar_wait_bounded(&mbar[it % kStages], (unsigned)(it / kStages) & 1u, kMbarWaitNs);
    }
  }
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  if (threadIdx.x < 32) tmem_dealloc_warp(base, kTmCols);
}

template <int NT>
static void launch_cheb3(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, int kb, int bf16,
                         const void* links, const float* scale, const float2* X, const float2* Z, const float2* S,
                         float2* Y, const double2* V, double2* W, const double* tcoef, int step, bool final_step,
                         cudaStream_t st) {
  const bool hz = Z != nullptr;
#define LAPH_CHEB3(LT, HZ, FIN)                                                                                \
  k_cheb_mrhs3<LT, HZ, FIN, NT><<<nblk, NT, 0, st>>>(pd, ps, start, np, kb, reinterpret_cast<const LT*>(links), \
                                                     scale, X, Z, S, Y, V, W, tcoef, step)
  if (bf16) {
    if (hz && final_step) LAPH_CHEB3(__nv_bfloat162, true, true);
    else if (hz) LAPH_CHEB3(__nv_bfloat162, true, false);
    else if (final_step) LAPH_CHEB3(__nv_bfloat162, false, true);
    else LAPH_CHEB3(__nv_bfloat162, false, false);
  } else {
    if (hz && final_step) LAPH_CHEB3(float2, true, true);
    else if (hz) LAPH_CHEB3(float2, true, false);
    else if (final_step) LAPH_CHEB3(float2, false, true);
    else LAPH_CHEB3(float2, false, false);
  }
#undef LAPH_CHEB3
}

template <int NT>
static void launch_cheb4(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, int kb, int bf16,
                         const void* links, const float* scale, const float2* X, const float2* Z, const float2* S,
                         float2* Y, const double2* V, double2* W, const double* tcoef, int step, bool final_step,
                         int lmax, int* err, cudaStream_t st) {
  const bool hz = Z != nullptr;
  const int stride = stage_stride(NT, lmax);
  const size_t smem = sizeof(float2) * (size_t)kStages * stride;
#define LAPH_CHEB4(LT, HZ, FIN)                                                                                   \
  k_cheb_mrhs4<LT, HZ, FIN, NT><<<nblk, NT, smem, st>>>(pd, ps, start, np, kb, reinterpret_cast<const LT*>(links), \
                                                        scale, X, Z, S, Y, V, W, tcoef, step, stride, err)
  if (bf16) {
    if (hz && final_step) LAPH_CHEB4(__nv_bfloat162, true, true);
    else if (hz) LAPH_CHEB4(__nv_bfloat162, true, false);
    else if (final_step) LAPH_CHEB4(__nv_bfloat162, false, true);
    else LAPH_CHEB4(__nv_bfloat162, false, false);
  } else {
    if (hz && final_step) LAPH_CHEB4(float2, true, true);
    else if (hz) LAPH_CHEB4(float2, true, false);
    else if (final_step) LAPH_CHEB4(float2, false, true);
    else LAPH_CHEB4(float2, false, false);
  }
#undef LAPH_CHEB4
}

// the staged variant's ring for the largest lattice it takes (L = 128)
template <int NT>
static int cheb4_attributes() {
  const int smem = (int)sizeof(float2) * kStages * stage_stride(NT, kStagedMaxL);
#define LAPH_ATTR(LT, HZ, FIN) \
  LAPH_CUDA_TRY(cudaFuncSetAttribute(k_cheb_mrhs4<LT, HZ, FIN, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem))
  LAPH_ATTR(float2, true, true);
  LAPH_ATTR(float2, true, false);
  LAPH_ATTR(float2, false, true);
  LAPH_ATTR(float2, false, false);
  LAPH_ATTR(__nv_bfloat162, true, true);
  LAPH_ATTR(__nv_bfloat162, true, false);
  LAPH_ATTR(__nv_bfloat162, false, true);
  LAPH_ATTR(__nv_bfloat162, false, false);
#undef LAPH_ATTR
  return LAPH_OK;
}

bool cheb_staged_ok(int L) { return L % 2 == 0 && L <= kStagedMaxL && kStagedNT % L == 0 && (L * L) % kStagedNT == 0; }

static void launch_cheb5(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, int kb, int bf16,
                         const void* links, const float* scale, const float2* X, const float2* Z, const float2* S,
                         float2* Y, const double2* V, double2* W, const double* tcoef, int step, bool final_step,
                         cudaStream_t st) {
  const bool hz = Z != nullptr;
#define LAPH_CHEB5(LT, HZ, FIN)                                                                          \
  k_cheb_mrhs5<LT, HZ, FIN><<<nblk, kBrickNT, 0, st>>>(pd, ps, start, np, kb, reinterpret_cast<const LT*>(links), \
                                                      scale, X, Z, S, Y, V, W, tcoef, step)
  if (bf16) {
    if (hz && final_step) LAPH_CHEB5(__nv_bfloat162, true, true);
    else if (hz) LAPH_CHEB5(__nv_bfloat162, true, false);
    else if (final_step) LAPH_CHEB5(__nv_bfloat162, false, true);
    else LAPH_CHEB5(__nv_bfloat162, false, false);
  } else {
    if (hz && final_step) LAPH_CHEB5(float2, true, true);
    else if (hz) LAPH_CHEB5(float2, true, false);
    else if (final_step) LAPH_CHEB5(float2, false, true);
    else LAPH_CHEB5(float2, false, false);
  }
#undef LAPH_CHEB5
}

template <int NT>
static void launch_cheb6(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, int kb, int bf16,
                         const void* links, const float* scale, const float2* X, const float2* Z, const float2* S,
                         float2* Y, const double2* V, double2* W, const double* tcoef, int step, bool final_step,
                         cudaStream_t st) {
  const bool hz = Z != nullptr;
  const size_t smem = sizeof(float2) * 2 * kPipeSlots * NT;
#define LAPH_CHEB6(LT, HZ, FIN)                                                                                   \
  k_cheb_mrhs6<LT, HZ, FIN, NT><<<nblk, NT, smem, st>>>(pd, ps, start, np, kb, reinterpret_cast<const LT*>(links), \
                                                        scale, X, Z, S, Y, V, W, tcoef, step)
  if (bf16) {
    if (hz && final_step) LAPH_CHEB6(__nv_bfloat162, true, true);
    else if (hz) LAPH_CHEB6(__nv_bfloat162, true, false);
    else if (final_step) LAPH_CHEB6(__nv_bfloat162, false, true);
    else LAPH_CHEB6(__nv_bfloat162, false, false);
  } else {
    if (hz && final_step) LAPH_CHEB6(float2, true, true);
    else if (hz) LAPH_CHEB6(float2, true, false);
    else if (final_step) LAPH_CHEB6(float2, false, true);
    else LAPH_CHEB6(float2, false, false);
  }
#undef LAPH_CHEB6
}

template <int NT>
static int cheb6_attributes() {
  const int smem = (int)sizeof(float2) * 2 * kPipeSlots * NT;
#define LAPH_ATTR(LT, HZ, FIN) \
  LAPH_CUDA_TRY(cudaFuncSetAttribute(k_cheb_mrhs6<LT, HZ, FIN, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem))
  LAPH_ATTR(float2, true, true);
  LAPH_ATTR(float2, true, false);
  LAPH_ATTR(float2, false, true);
  LAPH_ATTR(float2, false, false);
  LAPH_ATTR(__nv_bfloat162, true, true);
  LAPH_ATTR(__nv_bfloat162, true, false);
  LAPH_ATTR(__nv_bfloat162, false, true);
  LAPH_ATTR(__nv_bfloat162, false, false);
#undef LAPH_ATTR
  return LAPH_OK;
}

int cheb_variants_init() {
  LAPH_TRY(cheb4_attributes<kStagedNT>());
  LAPH_TRY(cheb6_attributes<64>());
  LAPH_TRY(cheb6_attributes<128>());
  LAPH_TRY(cheb6_attributes<256>());
  return LAPH_OK;
}

int cheb_variant_step(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, int kb, int bf16,
                      const void* links, const float* scale, const float2* X, const float2* Z, const float2* S,
                      float2* Y, const double2* V, double2* W, const double* tcoef, int step, bool final_step,
                      int variant, int tile, int lmax, int* err, cudaStream_t st) {
  if (variant == 5 && kb <= kCoefMax) {
    if (tile == 64)
      launch_cheb6<64>(pd, ps, start, np, nblk, kb, bf16, links, scale, X, Z, S, Y, V, W, tcoef, step, final_step, st);
    else if (tile == 256)
      launch_cheb6<256>(pd, ps, start, np, nblk, kb, bf16, links, scale, X, Z, S, Y, V, W, tcoef, step, final_step,
                        st);
    else
      launch_cheb6<128>(pd, ps, start, np, nblk, kb, bf16, links, scale, X, Z, S, Y, V, W, tcoef, step, final_step,
                        st);
    LAPH_CUDA_TRY(cudaGetLastError());
    return LAPH_OK;
  }
  if (variant == 4 && kb <= kCoefMax) {
    if (tile != kBrickNT || !cheb_staged_ok(lmax)) return LAPH_EINVAL;
    launch_cheb5(pd, ps, start, np, nblk, kb, bf16, links, scale, X, Z, S, Y, V, W, tcoef, step, final_step, st);
    LAPH_CUDA_TRY(cudaGetLastError());
    return LAPH_OK;
  }
  if (variant == 3 && kb <= kCoefMax) {
    if (tile != kStagedNT || !cheb_staged_ok(lmax) || err == nullptr) return LAPH_EINVAL;
    launch_cheb4<kStagedNT>(pd, ps, start, np, nblk, kb, bf16, links, scale, X, Z, S, Y, V, W, tcoef, step, final_step,
                            lmax, err, st);
    LAPH_CUDA_TRY(cudaGetLastError());
    return LAPH_OK;
  }
  if (variant == 2 && kb <= kCoefMax) {
    if (tile == 64)
      launch_cheb3<64>(pd, ps, start, np, nblk, kb, bf16, links, scale, X, Z, S, Y, V, W, tcoef, step, final_step, st);
    else if (tile == 256)
      launch_cheb3<256>(pd, ps, start, np, nblk, kb, bf16, links, scale, X, Z, S, Y, V, W, tcoef, step, final_step,
                        st);
    else
      launch_cheb3<128>(pd, ps, start, np, nblk, kb, bf16, links, scale, X, Z, S, Y, V, W, tcoef, step, final_step,
                        st);
    LAPH_CUDA_TRY(cudaGetLastError());
    return LAPH_OK;
  }
  return LAPH_EINVAL;
}

}  // namespace laph
