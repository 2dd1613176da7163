// filter.cu -- the multi-right-hand-side Chebyshev filter (lap_cheb_mrhs) and
// the other block stencils of the batched solver.
//
// lap_cheb_mrhs: one Chebyshev step on a block of k vectors of every active
// problem in one launch,
//     Y_j = a_j (c_hop hop(X_j) + c_diag X_j) + z_j Z_j + g_j S_j ,
// FP32 arithmetic on complex64 vectors, links FP32 or BF16 (+ FP32 per-site
// scale) reconstructed to FP32 in registers.  One thread owns one site and
// walks kb columns, so the 6 links a site needs (its 3 forward links and the
// 3 backward links U_mu(x-mu)) are read from HBM once per kb vectors and held
// in 108 registers; the vector reads of consecutive threads are consecutive
// site values (fully coalesced), neighbour reuse comes from L1/L2.  Inside
// each column the blocks (FP32 S and E ring, FP64 V, W, Y) are colour-major,
// element (site, c) at c*V3 + site, so every warp load is one dense 256-byte
// (FP32) or 512-byte (FP64) access; the solver converts to the reference's
// 3*site + colour order only on output.
// Per-column coefficients (a_j, z_j, g_j) come from a device table written by
// the Rayleigh-Ritz step, so every launch of an iteration is identical.
// Algorithmic bytes per site and vector: 24 (X) + 24 (S) + 24 (Z) + 24 (Y)
// plus (108 + 4) / kb for BF16 links; see the solver for the recurrence.
#include "batch.cuh"
#include "filter.cuh"
#include "stencil64cols.cuh"
#include "bulk.cuh"
#include "tmem.cuh"

#include <cuda_bf16.h>

namespace laph {

// ---------------------------------------------------------------- links ----
__device__ __forceinline__ float2 ld_lk(const float2* __restrict__ p, const float*, size_t i, int) { return __ldg(p + i); }
__device__ __forceinline__ float2 ld_lk(const __nv_bfloat162* __restrict__ p, const float* __restrict__ sc, size_t i,
                                        int site) {
  const float2 v = __bfloat1622float2(__ldg(p + i));
  const float s = __ldg(sc + site);
  return make_float2(v.x * s, v.y * s);
}

// FP64 site-minor links -> filter links (FP32, or BF16 with a per-site scale
// = max |element| over the site's 27 complex entries).
__global__ void k_pack_links(const ProbDesc* __restrict__ pd, const int* __restrict__ start, int np,
                             const double2* __restrict__ U64, float2* __restrict__ Uf32,
                             __nv_bfloat162* __restrict__ Ubf, float* __restrict__ scale, int bf16) {
  const int p = find_prob(start, np, blockIdx.x);
  const ProbDesc d = pd[p];
  const int s = (blockIdx.x - start[p]) * blockDim.x + threadIdx.x;
  if (s >= d.V3) return;
  const double2* U = U64 + d.u64;
  if (!bf16) {
    for (int e = 0; e < 27; ++e) {
      const double2 v = U[(size_t)e * d.V3 + s];
      Uf32[d.uf + (size_t)e * d.V3 + s] = make_float2((float)v.x, (float)v.y);
    }
    return;
  }
  double m = 0.0;
  for (int e = 0; e < 27; ++e) {
    const double2 v = U[(size_t)e * d.V3 + s];
    m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
  }
  const float scl = m > 0.0 ? (float)m : 1.0f;
  scale[d.sc + s] = scl;
  const double inv = 1.0 / (double)scl;
  for (int e = 0; e < 27; ++e) {
    const double2 v = U[(size_t)e * d.V3 + s];
    Ubf[d.uf + (size_t)e * d.V3 + s] = __floats2bfloat162_rn((float)(v.x * inv), (float)(v.y * inv));
  }
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

// ---------------------------------------------------------- the filter -----
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

template <typename LT, bool HAS_Z, bool FINAL>
__global__ void __launch_bounds__(128, 3)
    k_cheb_mrhs(const ProbDesc* __restrict__ pd, const ProbState* __restrict__ ps, const int* __restrict__ start, int np,
                int kb, const LT* __restrict__ links, const float* __restrict__ scale, const float2* __restrict__ Xp,
                const float2* __restrict__ Zp, const float2* __restrict__ Sp, float2* __restrict__ Yp,
                const double2* __restrict__ Vp, double2* __restrict__ Wp, const double* __restrict__ tcoef, int step) {
  const int p = find_prob(start, np, blockIdx.x);
  if (!ps[p].active) return;
  const ProbDesc d = pd[p];
  const int nst = (d.V3 + 127) >> 7;
  const int t = blockIdx.x - start[p];
  const int st = t % nst, cb = t / nst;
  const int s = st * 128 + threadIdx.x;
  if (s >= d.V3) return;
  const int j1 = min(cb * kb + kb, d.k);
  const int nlock = ps[p].nlock;
  if (FINAL) {
    // locked columns: W_j = V_j
    for (int j = cb * kb; j < min(j1, nlock); ++j) {
      const size_t i = (size_t)d.blk + (size_t)j * d.dim + s;
#pragma unroll
      for (int a = 0; a < 3; ++a) Wp[i + (size_t)a * d.V3] = __ldg(Vp + i + (size_t)a * d.V3);
    }
  }
  const int j0 = max(cb * kb, nlock);
  if (j0 >= j1) return;
  const Lat g{d.L, d.L * d.L, d.V3};
  int sx, sy, sz;
  site_xyz(g, s, sx, sy, sz);
  int up[3], dn[3];
#pragma unroll
  for (int mu = 0; mu < 3; ++mu) {
    up[mu] = nb_up(g, sx, sy, sz, mu);
    dn[mu] = nb_dn(g, sx, sy, sz, mu);
  }
  // 6 links in registers: forward U_mu(s), backward U_mu(s-mu)
  const LT* U = links + d.uf;
  const float* scl = scale + d.sc;
  float2 uf[3][9], ub[3][9];
#pragma unroll
  for (int mu = 0; mu < 3; ++mu)
#pragma unroll
    for (int e = 0; e < 9; ++e) {
      uf[mu][e] = ld_lk(U, scl, (size_t)(mu * 9 + e) * d.V3 + s, s);
      ub[mu][e] = ld_lk(U, scl, (size_t)(mu * 9 + e) * d.V3 + dn[mu], dn[mu]);
    }
  const double c_hop = ps[p].c_hop, c_diag = ps[p].c_diag;
  // coefficient table of this step: [step][0..2][k] = (a_j, z_j, g_j); the
  // final step also reads [step+1][0][k] = T_m / nu_m (see k_coef)
  const double* tc = tcoef + d.tc + (size_t)step * 3 * d.k;
  const size_t base = (size_t)d.blk;
  // One thread per CTA streams this tile's rows of X, S, Z (and V) for the
  // column kPrefetch ahead into L2 with bulk prefetches: no registers, no
  // shared memory, no waiting; the loads below then hit L2.
  const int s0 = st * 128, nsite = min(128, d.V3 - s0);
  const bool pf = threadIdx.x == 0 && (nsite % 2 == 0) && (d.dim % 2 == 0);
  auto prefetch = [&](int j) {
    if (!pf || j >= j1) return;
    const size_t col = base + (size_t)j * d.dim;
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
    const size_t col = base + (size_t)j * d.dim;
    const float2* x = Xp + col;
    float2 acc[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
#pragma unroll
    for (int mu = 0; mu < 3; ++mu) {
      float2 xu[3], xd[3];
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        xu[b] = __ldg(x + (size_t)b * d.V3 + up[mu]);
        xd[b] = __ldg(x + (size_t)b * d.V3 + dn[mu]);
      }
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          cfmaf(acc[a], uf[mu][3 * a + b], xu[b]);
          cfmacf(acc[a], ub[mu][3 * b + a], xd[b]);
        }
    }
    const double aj = __ldg(tc + j);
    const float a_h = (float)(aj * c_hop), a_d = (float)(aj * c_diag);
    const float zc = (float)__ldg(tc + d.k + j);
    const float gj = (float)__ldg(tc + 2 * d.k + j);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const size_t i = col + (size_t)a * d.V3 + s;  // colour-major FP32 buffers
      const float2 xs = __ldg(x + (size_t)a * d.V3 + s);
      const float2 ss = __ldg(Sp + i);
      float2 r;
      r.x = fmaf(a_h, acc[a].x, fmaf(a_d, xs.x, gj * ss.x));
      r.y = fmaf(a_h, acc[a].y, fmaf(a_d, xs.y, gj * ss.y));
      if (HAS_Z) {
        const float2 zz = __ldg(Zp + i);
        r.x = fmaf(zc, zz.x, r.x);
        r.y = fmaf(zc, zz.y, r.y);
      }
      if (FINAL) {
        // W = T_m(theta_B) V + E_m in FP64 (FP64 blocks are colour-major too)
        const double tm = __ldg(tc + (size_t)3 * d.k + j);
        const size_t iv = col + (size_t)a * d.V3 + s;
        const double2 v = __ldg(Vp + iv);
        Wp[iv] = make_double2(fma(tm, v.x, (double)r.x), fma(tm, v.y, (double)r.y));
      } else {
        Yp[i] = r;
      }
    }
  }
}

// Variant of the same step for column blocks kb <= kCoefMax (the default): the
// CTA first converts this step's coefficients of its columns to FP32
// (a c_hop, a c_diag, z, g) in shared memory, so the column loop reads one
// broadcast float4 instead of three FP64 loads and four conversions per
// thread; and the site's three backward links live in shared memory (27.6 KB
// per CTA, each thread its own column) instead of registers, which takes the
// kernel from 168 to 128 registers and from 12 to 16 warps per SM (+12%
// filter throughput; also moving one forward direction there, for 20 warps,
// measured 5% slower).  The hop runs as packed fma.rn.f32x2 on (re, im) pairs:
// half the FMA instructions of the scalar form, +1%.  (Software-pipelining the loop over column pairs, with the 27
// vector values of column j+1 in flight while column j is computed, needs
// ~250 registers, halves residency to 2 CTAs per SM and measured no faster.)
constexpr int kCoefMax = 64;
struct ChebCol {
  float2 xu[3][3], xd[3][3], xs[3], ss[3], zz[3];
};

// NT sites (threads) per CTA, the tile the autotuner picks (64, 128 or 256);
// 16 warps per SM at 128 registers whichever NT.
template <typename LT, bool HAS_Z, bool FINAL, int NT, bool HAS_S = true>
__global__ void __launch_bounds__(NT, 512 / NT)
    k_cheb_mrhs2(const ProbDesc* __restrict__ pd, const ProbState* __restrict__ ps, const int* __restrict__ start,
                 int np, int kb, const LT* __restrict__ links, const float* __restrict__ scale,
                 const float2* __restrict__ Xp, const float2* __restrict__ Zp, const float2* __restrict__ Sp,
                 float2* __restrict__ Yp, const double2* __restrict__ Vp, double2* __restrict__ Wp,
                 const double* __restrict__ tcoef, int step) {
  const int p = find_prob(start, np, blockIdx.x);
  if (!ps[p].active) return;
  const ProbDesc d = pd[p];
  const int nst = (d.V3 + NT - 1) / NT;
  const int t = blockIdx.x - start[p];
  const int st = t % nst, cb = t / nst;
  const int s = st * NT + threadIdx.x;
  const bool valid = s < d.V3;
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
  if (j0 >= j1) return;  // uniform over the CTA
  __shared__ float4 cf[kCoefMax];
  __shared__ double ctm[kCoefMax];
  {
    const double c_hop = ps[p].c_hop, c_diag = ps[p].c_diag;
    const double* tc = tcoef + d.tc + (size_t)step * 3 * d.k;
    for (int j = j0 + (int)threadIdx.x; j < j1; j += NT) {
      const double a = tc[j];
      cf[LAPH_IX(j - j0, kCoefMax)] = make_float4((float)(a * c_hop), (float)(a * c_diag), (float)tc[d.k + j], (float)tc[2 * d.k + j]);
      if (FINAL) ctm[LAPH_IX(j - j0, kCoefMax)] = tc[(size_t)3 * d.k + j];
    }
  }
  __syncthreads();
  if (!valid) return;
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
  // forward links in registers (54), backward links U_mu(s - mu) in shared
  // memory (dynamic, 27 x NT float2), each thread reading only its own column
  // of sUb (no sharing, no barrier): 128 registers instead of 168, 16 warps per SM
  extern __shared__ float2 sUb_dyn[];
  float2 (*sUb)[NT] = reinterpret_cast<float2 (*)[NT]>(sUb_dyn);
  float2 uf[3][9];
#pragma unroll
  for (int mu = 0; mu < 3; ++mu)
#pragma unroll
    for (int e = 0; e < 9; ++e) {
      uf[mu][e] = ld_lk(U, scl, (size_t)(mu * 9 + e) * d.V3 + s, s);
      float2 bwl = ld_lk(U, scl, (size_t)(mu * 9 + e) * d.V3 + dn[mu], dn[mu]);
      bwl.y = -bwl.y;  // stored conjugated for the packed FP32x2 hop
      sUb[mu * 9 + e][threadIdx.x] = bwl;
    }
  const size_t base = (size_t)d.blk;
  const int s0 = st * NT, nsite = min(NT, d.V3 - s0);
  const bool pf = threadIdx.x == 0 && (nsite % 2 == 0) && (d.dim % 2 == 0);
  auto prefetch = [&](int j) {
    if (!pf || j >= j1) return;
    const size_t col = base + (size_t)j * d.dim;
    const unsigned bytes = 8u * nsite;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      l2_prefetch(Xp + col + (size_t)c * d.V3 + s0, bytes);
      if (HAS_S) l2_prefetch(Sp + col + (size_t)c * d.V3 + s0, bytes);
      if (HAS_Z) l2_prefetch(Zp + col + (size_t)c * d.V3 + s0, bytes);
    }
    if (FINAL)
#pragma unroll
      for (int c = 0; c < 3; ++c) l2_prefetch(Vp + col + (size_t)c * d.V3 + s0, 2 * bytes);
  };
  auto fetch = [&](int j, ChebCol& c) {
    const size_t col = base + (size_t)j * d.dim;
    const float2* x = Xp + col;
#pragma unroll
    for (int mu = 0; mu < 3; ++mu)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        c.xu[mu][b] = __ldg(x + (size_t)b * d.V3 + up[mu]);
        c.xd[mu][b] = __ldg(x + (size_t)b * d.V3 + dn[mu]);
      }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      c.xs[a] = __ldg(x + (size_t)a * d.V3 + s);
      c.ss[a] = HAS_S ? __ldg(Sp + col + (size_t)a * d.V3 + s) : make_float2(0.f, 0.f);
      if (HAS_Z) c.zz[a] = __ldg(Zp + col + (size_t)a * d.V3 + s);
    }
  };
  auto compute = [&](int j, const ChebCol& c) {
    float2 acc[3];
    // packed FP32x2: with u = (re, im), P += (x.re, x.re) u and T += (x.im, x.im) u
    // give u x = (P.x - T.y, P.y + T.x); backward links are stored conjugated
    unsigned long long P[3] = {0ull, 0ull, 0ull}, T[3] = {0ull, 0ull, 0ull};
#pragma unroll
    for (int mu = 0; mu < 3; ++mu)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const unsigned long long ur = pk2(c.xu[mu][b].x, c.xu[mu][b].x), ui = pk2(c.xu[mu][b].y, c.xu[mu][b].y);
        const unsigned long long dr = pk2(c.xd[mu][b].x, c.xd[mu][b].x), di = pk2(c.xd[mu][b].y, c.xd[mu][b].y);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const unsigned long long lf = pk2(uf[mu][3 * a + b].x, uf[mu][3 * a + b].y);
          const float2 bw = sUb[mu * 9 + 3 * b + a][threadIdx.x];
          const unsigned long long lb = pk2(bw.x, bw.y);
          ffma2(P[a], ur, lf);
          ffma2(T[a], ui, lf);
          ffma2(P[a], dr, lb);
          ffma2(T[a], di, lb);
        }
      }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float2 pp = unpk2(P[a]), tt = unpk2(T[a]);
      acc[a] = make_float2(pp.x - tt.y, pp.y + tt.x);
    }
    const float4 q = cf[LAPH_IX(j - j0, kCoefMax)];  // (a c_hop, a c_diag, z, g)
    const size_t col = base + (size_t)j * d.dim;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float2 r;
      r.x = fmaf(q.x, acc[a].x, fmaf(q.y, c.xs[a].x, q.w * c.ss[a].x));
      r.y = fmaf(q.x, acc[a].y, fmaf(q.y, c.xs[a].y, q.w * c.ss[a].y));
      if (HAS_Z) {
        r.x = fmaf(q.z, c.zz[a].x, r.x);
        r.y = fmaf(q.z, c.zz[a].y, r.y);
      }
      if (FINAL) {
        const size_t iv = col + (size_t)a * d.V3 + s;
        const double2 v = __ldg(Vp + iv);
        const double tm = ctm[LAPH_IX(j - j0, kCoefMax)];
        Wp[iv] = make_double2(fma(tm, v.x, (double)r.x), fma(tm, v.y, (double)r.y));
      } else {
        Yp[col + (size_t)a * d.V3 + s] = r;
      }
    }
  };
#pragma unroll 1
  for (int j = j0; j < min(j1, j0 + kPrefetch); ++j) prefetch(j);
  ChebCol A;
#pragma unroll 1
  for (int j = j0; j < j1; ++j) {
    prefetch(j + kPrefetch);
    fetch(j, A);
    compute(j, A);
  }
}

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

// The start of a direct pass (ProbState::direct): S = V in FP32, for the
// unlocked columns of the problems that filter directly (the others keep the
// S the residual kernel wrote).  Same grid as the filter: tile sites x kb
// columns per CTA.
__global__ void k_direct_start(const ProbDesc* __restrict__ pd, const ProbState* __restrict__ ps,
                               const int* __restrict__ start, int np, int kb, int tile,
                               const double2* __restrict__ Vp, float2* __restrict__ Sp) {
  const int p = find_prob(start, np, blockIdx.x);
  if (!ps[p].active || !ps[p].direct) return;
  const ProbDesc d = pd[p];
  const int nst = (d.V3 + tile - 1) / tile;
  const int t = blockIdx.x - start[p];
  const int st = t % nst, cb = t / nst;
  const int j0 = max(cb * kb, ps[p].nlock), j1 = min(cb * kb + kb, d.k);
  for (int sl = threadIdx.x; sl < tile; sl += blockDim.x) {
    const int s = st * tile + sl;
    if (s >= d.V3) break;
    for (int j = j0; j < j1; ++j) {
      const size_t i = (size_t)d.blk + (size_t)j * d.dim + s;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const double2 v = __ldg(Vp + i + (size_t)a * d.V3);
        Sp[i + (size_t)a * d.V3] = make_float2((float)v.x, (float)v.y);
      }
    }
  }
}

// ------------------------------------------------ FP64 block stencil: A W --
// Y_j = (-Delta) W_j = 6 W_j - hop(W_j), FP64; CTA = 128 sites x a block of
// kColsFP64 columns (stencil64cols.cuh).
__global__ void __launch_bounds__(128, 3) k_neglap64_batch(const ProbDesc* __restrict__ pd, const ProbState* __restrict__ ps,
                                                        const int* __restrict__ start, int np,
                                                        const double2* __restrict__ U64, const double2* __restrict__ Wp,
                                                        double2* __restrict__ Yp) {
  const int p = find_prob(start, np, blockIdx.x);
  if (!ps[p].active) return;
  const ProbDesc d = pd[p];
  const int nst = (d.V3 + kSites64 - 1) / kSites64;
  const int t = blockIdx.x - start[p];
  const int st = t % nst, cb = t / nst;
  if ((cb + 1) * kColsFP64 <= ps[p].c0) return;  // frozen columns: Y not needed
  const int s = st * kSites64 + threadIdx.x;
  if (s >= d.V3) return;
  const Lat g{d.L, d.L * d.L, d.V3};
  int sx, sy, sz, up[3], dn[3];
  site_xyz(g, s, sx, sy, sz);
#pragma unroll
  for (int mu = 0; mu < 3; ++mu) {
    up[mu] = nb_up(g, sx, sy, sz, mu);
    dn[mu] = nb_dn(g, sx, sy, sz, mu);
  }
  extern __shared__ double2 s64[];
  double2 (*sUb)[kSites64] = reinterpret_cast<double2 (*)[kSites64]>(s64);
  Links64 l;
  load_links64(U64 + d.u64, g, s, dn, l, sUb);
  const int j1 = min(d.k, (cb + 1) * kColsFP64);
#pragma unroll 1
  for (int j = cb * kColsFP64; j < j1; ++j) {
    const size_t col = (size_t)d.blk + (size_t)j * d.dim;
    const double2* x = Wp + col;
    double2 acc[3];
    hop64_col(l, sUb, d.V3, up, dn, x, acc);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double2 xs = __ldg(x + (size_t)a * d.V3 + s);
      Yp[col + (size_t)a * d.V3 + s] = make_double2(6.0 * xs.x - acc[a].x, 6.0 * xs.y - acc[a].y);
    }
  }
}

// ------------------------------------------------------ random start block -
__device__ __forceinline__ uint64_t mix64d(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
__global__ void k_random_block(const ProbDesc* __restrict__ pd, const int* __restrict__ start, int np,
                               double2* __restrict__ W, uint64_t seed) {
  const int p = find_prob(start, np, blockIdx.x);
  const ProbDesc d = pd[p];
  const long long i = (long long)(blockIdx.x - start[p]) * blockDim.x + threadIdx.x;
  const long long n = (long long)d.dim * d.k;
  if (i >= n) return;
  uint64_t st = seed * 0x9E3779B97F4A7C15ULL + ((uint64_t)p << 40) + (uint64_t)i * 0xD1B54A32D192ED03ULL;
  const double u1 = ((mix64d(st + 0x9E3779B97F4A7C15ULL) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  const double u2 = ((mix64d(st + 0x3C6EF372FE94F82AULL) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  const double r = sqrt(-2.0 * log(u1));
  double sn, cs;
  sincospi(2.0 * u2, &sn, &cs);
  W[d.blk + i] = make_double2(r * cs, r * sn);
}

// ------------------------------------------------------------- launchers ---
int pack_links(const ProbDesc* pd, const int* start, int np, int nblk, const double2* U64, float2* Uf32, void* Ubf,
               float* scale, int bf16, cudaStream_t st) {
  k_pack_links<<<nblk, 128, 0, st>>>(pd, start, np, U64, Uf32, reinterpret_cast<__nv_bfloat162*>(Ubf), scale, bf16);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}

template <int NT>
static void launch_cheb2(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, int kb, int bf16,
                         const void* links, const float* scale, const float2* X, const float2* Z, const float2* S,
                         float2* Y, const double2* V, double2* W, const double* tcoef, int step, bool final_step,
                         bool no_s, cudaStream_t st) {
  const bool hz = Z != nullptr;
  const size_t smem = sizeof(float2) * 27 * NT;
#define LAPH_CHEB2(LT, HZ, FIN)                                                                                   \
  k_cheb_mrhs2<LT, HZ, FIN, NT><<<nblk, NT, smem, st>>>(pd, ps, start, np, kb, reinterpret_cast<const LT*>(links), \
                                                        scale, X, Z, S, Y, V, W, tcoef, step)
#define LAPH_CHEB2N(LT, FIN)                                                                                      \
  k_cheb_mrhs2<LT, true, FIN, NT, false><<<nblk, NT, smem, st>>>(                                                  \
      pd, ps, start, np, kb, reinterpret_cast<const LT*>(links), scale, X, Z, S, Y, V, W, tcoef, step)
  if (no_s && hz) {  // a step of a direct pass past its second: the S coefficient is 0
    if (bf16) {
      if (final_step) LAPH_CHEB2N(__nv_bfloat162, true);
      else LAPH_CHEB2N(__nv_bfloat162, false);
    } else {
      if (final_step) LAPH_CHEB2N(float2, true);
      else LAPH_CHEB2N(float2, false);
    }
    return;
  }
#undef LAPH_CHEB2N
  if (bf16) {
    if (hz && final_step) LAPH_CHEB2(__nv_bfloat162, true, true);
    else if (hz) LAPH_CHEB2(__nv_bfloat162, true, false);
    else if (final_step) LAPH_CHEB2(__nv_bfloat162, false, true);
    else LAPH_CHEB2(__nv_bfloat162, false, false);
  } else {
    if (hz && final_step) LAPH_CHEB2(float2, true, true);
    else if (hz) LAPH_CHEB2(float2, true, false);
    else if (final_step) LAPH_CHEB2(float2, false, true);
    else LAPH_CHEB2(float2, false, false);
  }
#undef LAPH_CHEB2
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

template <int NT>
static int cheb2_attributes() {
  const int smem = (int)sizeof(float2) * 27 * NT;
#define LAPH_ATTR(LT, HZ, FIN) \
  LAPH_CUDA_TRY(cudaFuncSetAttribute(k_cheb_mrhs2<LT, HZ, FIN, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem))
  LAPH_ATTR(float2, true, true);
  LAPH_ATTR(float2, true, false);
  LAPH_ATTR(float2, false, true);
  LAPH_ATTR(float2, false, false);
  LAPH_ATTR(__nv_bfloat162, true, true);
  LAPH_ATTR(__nv_bfloat162, true, false);
  LAPH_ATTR(__nv_bfloat162, false, true);
  LAPH_ATTR(__nv_bfloat162, false, false);
#undef LAPH_ATTR
#define LAPH_ATTRN(LT, FIN)                                                                                  \
  LAPH_CUDA_TRY(cudaFuncSetAttribute(k_cheb_mrhs2<LT, true, FIN, NT, false>,                               \
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, smem))
  LAPH_ATTRN(float2, true);
  LAPH_ATTRN(float2, false);
  LAPH_ATTRN(__nv_bfloat162, true);
  LAPH_ATTRN(__nv_bfloat162, false);
#undef LAPH_ATTRN
  return LAPH_OK;
}

// the 256-site tile keeps 55 KB of backward links in dynamic shared memory
int cheb_init() {
  LAPH_TRY(cheb2_attributes<64>());
  LAPH_TRY(cheb2_attributes<128>());
  LAPH_TRY(cheb2_attributes<256>());
  LAPH_TRY(cheb4_attributes<kStagedNT>());
  LAPH_TRY(cheb6_attributes<64>());
  LAPH_TRY(cheb6_attributes<128>());
  LAPH_TRY(cheb6_attributes<256>());
  return LAPH_OK;
}

int cheb_step(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, int kb, int bf16,
              const void* links, const float* scale, const float2* X, const float2* Z, const float2* S, float2* Y,
              const double2* V, double2* W, const double* tcoef, int step, bool final_step, int variant, int tile,
              int lmax, int* err, bool no_s, cudaStream_t st) {
  const bool hz = Z != nullptr;
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
  if (variant >= 1 && kb <= kCoefMax) {
    if (tile == 64)
      launch_cheb2<64>(pd, ps, start, np, nblk, kb, bf16, links, scale, X, Z, S, Y, V, W, tcoef, step, final_step,
                       no_s, st);
    else if (tile == 256)
      launch_cheb2<256>(pd, ps, start, np, nblk, kb, bf16, links, scale, X, Z, S, Y, V, W, tcoef, step, final_step,
                        no_s, st);
    else
      launch_cheb2<128>(pd, ps, start, np, nblk, kb, bf16, links, scale, X, Z, S, Y, V, W, tcoef, step, final_step,
                        no_s, st);
    LAPH_CUDA_TRY(cudaGetLastError());
    return LAPH_OK;
  }
#define LAPH_CHEB(LT, HZ, FIN)                                                                                  \
  k_cheb_mrhs<LT, HZ, FIN><<<nblk, 128, 0, st>>>(pd, ps, start, np, kb, reinterpret_cast<const LT*>(links), scale, \
                                                 X, Z, S, Y, V, W, tcoef, step)
  if (bf16) {
    if (hz && final_step) LAPH_CHEB(__nv_bfloat162, true, true);
    else if (hz) LAPH_CHEB(__nv_bfloat162, true, false);
    else if (final_step) LAPH_CHEB(__nv_bfloat162, false, true);
    else LAPH_CHEB(__nv_bfloat162, false, false);
  } else {
    if (hz && final_step) LAPH_CHEB(float2, true, true);
    else if (hz) LAPH_CHEB(float2, true, false);
    else if (final_step) LAPH_CHEB(float2, false, true);
    else LAPH_CHEB(float2, false, false);
  }
#undef LAPH_CHEB
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}

int direct_start(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, int kb, int tile,
                 const double2* V, float2* S, cudaStream_t st) {
  k_direct_start<<<nblk, 128, 0, st>>>(pd, ps, start, np, kb, tile, V, S);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}

int neglap64_init() {
  LAPH_CUDA_TRY(cudaFuncSetAttribute(k_neglap64_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, kStencil64Smem));
  return LAPH_OK;
}

int neglap64_batch(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, const double2* U64,
                   const double2* W, double2* Y, cudaStream_t st) {
  k_neglap64_batch<<<nblk, kSites64, kStencil64Smem, st>>>(pd, ps, start, np, U64, W, Y);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}

int random_block(const ProbDesc* pd, const int* start, int np, int nblk, double2* W, uint64_t seed, cudaStream_t st) {
  k_random_block<<<nblk, 256, 0, st>>>(pd, start, np, W, seed);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}

}  // namespace laph
