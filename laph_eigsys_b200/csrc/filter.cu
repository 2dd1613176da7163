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
#include "filter_common.cuh"
#include "filter_variants.cuh"
#include "stencil64cols.cuh"

#include <cuda_bf16.h>

namespace laph {

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
  return cheb_variants_init();
}

int cheb_step(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, int kb, int bf16,
              const void* links, const float* scale, const float2* X, const float2* Z, const float2* S, float2* Y,
              const double2* V, double2* W, const double* tcoef, int step, bool final_step, int variant, int tile,
              int lmax, int* err, bool no_s, cudaStream_t st) {
  const bool hz = Z != nullptr;
  if (variant >= 2 && variant <= 5 && kb <= kCoefMax)
    return cheb_variant_step(pd, ps, start, np, nblk, kb, bf16, links, scale, X, Z, S, Y, V, W, tcoef, step, final_step,
                             variant, tile, lmax, err, st);
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
