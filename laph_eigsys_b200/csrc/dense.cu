// dense.cu -- FP64 dense block operations of the batched solver:
//   k_gram        [G | H] = W^H [W | Y]  (partials over row chunks)
//   k_gram_reduce fixed-order sum of the partials, Hermitian completion
//   k_small       per problem: column scaling, Cholesky, triangular inverse,
//                 projected Hermitian matrix, Jacobi eigensolve, sort, C,
//                 next Chebyshev window and coefficient table
//   k_rotate      V = W C
//   k_residual64  R = (-Delta) V - V diag(theta) (FP64 stencil), S = -2 c_hop R
//                 (FP32), residual partial sums
//   k_resid       residual norms, convergence mask
// Columns [0, c0) of a problem (whole tiles of locked Ritz vectors) are frozen:
// the Gram skips frozen x frozen tiles, the small problem projects the active
// block against them, and the rotation and residual write active columns only.
// These replace SLEPc's BV orthogonalisation and DS dense eigensolve inside
// EPSSolve (src/ev_ts.cpp:263).  tcgen05 has no FP64 kind, so the Gram and the
// rotation run on the FP64 tensor path of mma.sync (four real MMAs per complex
// product): at the same peak as the FP64 FMA pipe, but one instruction per 256
// FMAs (m8n8k4, the rotation) or 2048 (m16n8k16, the Gram), which measured
// 7-10% faster for each kernel than FMA, and the Gram another 9% on m16n8k16.
#include "batch.cuh"
#include "dense.cuh"
#include "filter.cuh"
#include "stencil64cols.cuh"

namespace laph {

// d(8x8, 2 per thread) += a(8x4, 1 per thread) b(4x8, 1 per thread), FP64 tensor MMA.
// Not volatile: a pure function of its operands, so the compiler may schedule
// it; the callers issue the MMAs of one k-step accumulator-major (all tiles'
// first product, then all tiles' second, ...) so that consecutive MMAs never
// feed the same accumulator and the tensor pipe does not wait on its latency.
__device__ __forceinline__ void dmma884(double (&acc)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(acc[0]), "+d"(acc[1])
      : "d"(a), "d"(b));
}
// d(16x8, 4 per thread) += a(16x16, 8 per thread) b(16x8, 4 per thread), FP64 tensor MMA: the same peak as
// m8n8k4 (37.1 TFLOP/s measured for both on this part) with an eighth of the instructions.  Fragments, g =
// lane / 4, t = lane % 4: a[r] = A(g + 8 (r & 1), t + 4 (r >> 1)); b[r] = B(t + 4 r, g); d[0..1] = D(g, 2t + {0,1}),
// d[2..3] = D(g + 8, 2t + {0,1}).
__device__ __forceinline__ void dmma16816(double (&d)[4], const double (&a)[8], const double (&b)[4]) {
  asm("mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
      "{%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]), "d"(b[1]),
        "d"(b[2]), "d"(b[3]));
}

// ------------------------------------------------------------------ Gram ---
// CTA: 64 threads, output tiles G[ti,tj] = W_ti^H W_tj and H[ti,tj] = W_ti^H Y_tj
// (32 x 32 each, as 2 x 4 m16n8k16 tiles; warp 0 forms G, warp 1 H), over the rows of one chunk; the
// W_ti tile is staged once for both products.  Rows arrive through a
// two-stage cp.async ring (dynamic shared memory [stage][A|W|Y][col][GP], row q of column c at
// c GP + (q ^ 4 (c & 1)): the 16-byte fragment reads of a quarter warp, two columns of one parity pair,
// then fall on eight different bank groups),
// so the next 16 rows load while the current 16 are multiplied.
constexpr int GT = 32, GK = 16, GP = GK;
__device__ __forceinline__ int gsw(int c, int q) { return c * GP + (q ^ ((c & 1) << 2)); }
constexpr int kGramSmem = 2 * 3 * GT * GP * (int)sizeof(double2);

__global__ void __launch_bounds__(64) k_gram(const ProbDesc* __restrict__ pd, const ProbState* __restrict__ ps,
                                             const int* __restrict__ start, int np, int chunk_rows,
                                             const double2* __restrict__ W, const double2* __restrict__ Y,
                                             double2* __restrict__ gpart) {
  const int p = find_prob(start, np, blockIdx.x);
  if (!ps[p].active) return;
  const ProbDesc d = pd[p];
  const int T = d.k / GT;
  const int npair = T * (T + 1) / 2;
  int t = blockIdx.x - start[p];
  const int chunk = t / npair;
  const int pair = t - chunk * npair;
  int pr = pair, ti = 0;
  while (pr >= T - ti) {
    pr -= T - ti;
    ++ti;
  }
  const int tj = LAPH_IX(ti + pr, T);
  if ((tj + 1) * GT <= ps[p].c0) return;  // both tiles frozen: not needed
  const double2* A = W + d.blk + (size_t)(ti * GT) * d.dim;
  const double2* BW = W + d.blk + (size_t)(tj * GT) * d.dim;
  const double2* BY = Y + d.blk + (size_t)(tj * GT) * d.dim;
  const int r0 = chunk * chunk_rows, r1 = min(d.dim, r0 + chunk_rows);
  extern __shared__ double2 gsm[];
  // thread -> (column c, row q) of each staged 32 x 16 slab: 16 threads per column, 256 B contiguous
  auto load = [&](int r, int b) {
    double2* s = gsm + b * 3 * GT * GP;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int idx = threadIdx.x + 64 * e;
      const int c = idx >> 4, q = idx & 15;
      const int row = r + q;
      const bool ok = row < r1;
      const size_t off = (size_t)c * d.dim + (ok ? row : 0);
      cp_async16(s + LAPH_IX(gsw(c, q), GT * GP), A + off, ok);
      cp_async16(s + gsw(GT + c, q), BW + off, ok);
      cp_async16(s + gsw(2 * GT + c, q), BY + off, ok);
    }
    cp_async_commit();
  };
  // FP64 tensor path: warp 0 forms G = W_ti^H W_tj, warp 1 H = W_ti^H Y_tj, each
  // as 2 x 4 tiles of m16n8k16 (one MMA per tile and stage of 16 rows);
  // conj(w) b = (wr br + wi bi) + i (wr bi - wi br), the last as wi (-br)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t4 = lane & 3;
  double accr[2][4][4], acci[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) accr[i][j][e] = acci[i][j][e] = 0.0;
  const int nstep = (r1 - r0 + GK - 1) / GK;
  // On a diagonal tile pair (ti == tj) the reduction keeps only the upper
  // triangle (G and H are Hermitian): the 16x8 tiles entirely below the
  // diagonal (rows 16-31 x columns 0-15) are skipped, 2 of 8 per warp.
  const bool diag = ti == tj;
  load(r0, 0);
  for (int it = 0; it < nstep; ++it) {
    const int b = it & 1;
    if (it + 1 < nstep) {
      load(r0 + (it + 1) * GK, b ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const double2* sA = gsm + b * 3 * GT * GP;
    const double2* sB = sA + (1 + warp) * GT * GP;  // W_tj or Y_tj
    // A fragments (m16 x k16, row = column of W_ti, k = row of the stage): a[r] at (g + 8 (r & 1), t4 + 4 (r >> 1))
    double ar[2][8], ai[2][8];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const double2 a = sA[gsw(16 * i + g + 8 * (r & 1), t4 + 4 * (r >> 1))];
        ar[i][r] = a.x;
        ai[i][r] = a.y;
      }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      // B fragment (k16 x n8): b[r] at (t4 + 4 r, g)
      double br[4], bi[4], bn[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const double2 v = sB[gsw(8 * j + g, t4 + 4 * r)];
        br[r] = v.x;
        bi[r] = v.y;
        bn[r] = -v.x;
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
        if (!diag || !(i == 1 && j < 2)) dmma16816(accr[i][j], ar[i], br);
#pragma unroll
      for (int i = 0; i < 2; ++i)
        if (!diag || !(i == 1 && j < 2)) dmma16816(acci[i][j], ar[i], bi);
#pragma unroll
      for (int i = 0; i < 2; ++i)
        if (!diag || !(i == 1 && j < 2)) dmma16816(accr[i][j], ai[i], bi);
#pragma unroll
      for (int i = 0; i < 2; ++i)
        if (!diag || !(i == 1 && j < 2)) dmma16816(acci[i][j], ai[i], bn);
    }
    __syncthreads();
  }
  // partial layout: [chunk][which][pair][32*32]; C fragment rows g (+8), columns 2 t4 + {0, 1}
  double2* o = gpart + d.gp + ((size_t)(chunk * 2 + warp) * npair + pair) * (GT * GT);
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int rb = 2 * i + h;  // 8-row block of the output
        if (diag && rb > j) continue;
#pragma unroll
        for (int e = 0; e < 2; ++e)
          o[(16 * i + 8 * h + g) * GT + 8 * j + 2 * t4 + e] = make_double2(accr[i][j][2 * h + e], acci[i][j][2 * h + e]);
      }
}


// Sum partials (fixed order) and complete the Hermitian matrices G, H
// (column-major k x k at kk and kk + k*k).
__global__ void k_gram_reduce(const ProbDesc* __restrict__ pd, const ProbState* __restrict__ ps,
                              const int* __restrict__ start, int np, const double2* __restrict__ gpart,
                              double2* __restrict__ GH) {
  const int p = find_prob(start, np, blockIdx.x);
  if (!ps[p].active) return;
  const ProbDesc d = pd[p];
  const int T = d.k / GT, npair = T * (T + 1) / 2;
  const int e = (blockIdx.x - start[p]) * blockDim.x + threadIdx.x;
  if (e >= 2 * npair * GT * GT) return;
  const int tile = e / (GT * GT), w = e - tile * GT * GT;
  const int which = tile / npair;
  int pr = tile - which * npair, ti = 0;
  while (pr >= T - ti) {
    pr -= T - ti;
    ++ti;
  }
  const int tj = ti + pr;
  if ((tj + 1) * GT <= ps[p].c0) return;  // frozen tile pair: not computed
  double2 s = make_double2(0.0, 0.0);
  for (int c = 0; c < d.nchunk; ++c) s = cadd(s, gpart[d.gp + ((size_t)(c * 2 + which) * npair + tile - which * npair) * (GT * GT) + w]);
  const int i = ti * GT + w / GT, j = tj * GT + w % GT;
  double2* M = GH + d.kk + (size_t)which * d.k * d.k;
  if (ti == tj) {
    // diagonal tile holds both triangles; keep the upper one and mirror it
    if (i <= j) {
      if (i == j) s.y = 0.0;
      M[i + (size_t)j * d.k] = s;
      M[j + (size_t)i * d.k] = cconj(s);
    }
  } else {
    M[i + (size_t)j * d.k] = s;
    M[j + (size_t)i * d.k] = cconj(s);
  }
}

// ------------------------------------------------------------ small dense --
// One CTA (1024 threads) per active problem.  Work arrays (column-major k x k)
// at kk: [0] G -> C, [1] H, [2] Minv, [3] T1 / Q, [4] Ht.
__device__ __forceinline__ double2& at(double2* M, int k, int i, int j) { return M[i + (size_t)j * k]; }

__global__ void __launch_bounds__(1024) k_small(const ProbDesc* __restrict__ pd, ProbState* __restrict__ ps,
                                                double2* __restrict__ KK, double* __restrict__ theta,
                                                double* __restrict__ tcoef, double* __restrict__ scol,
                                                double* __restrict__ dwork, int first_iter, int fixed_cut,
                                                int max_sweeps, unsigned long long* __restrict__ tstamp) {
  const int p = blockIdx.x;
  if (!ps[p].active) return;
  // phase boundaries (global timer, ns) for the solver's trace: [p][0..6]
  auto stamp = [&](int ph) {
    if (threadIdx.x == 0) {
      unsigned long long t;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
      tstamp[p * kSmallPhases + ph] = t;
    }
  };
  stamp(0);
  const ProbDesc d = pd[p];
  const int k = d.k, tid = threadIdx.x, nt = blockDim.x;
  // Locked columns [0, c0) (a multiple of the tile width) stay as they are: the
  // Rayleigh-Ritz runs on the active block a = [c0, k), with W_a projected
  // against the locked Ritz vectors V_l (= W_l).  n = k - c0; every matrix
  // below keeps the leading dimension k.
  const int c0 = ps[p].c0, n = k - c0;
  const size_t kk2 = (size_t)k * k;
  double2* G = KK + d.kk;
  double2* H = G + kk2;
  double2* Mi = G + 2 * kk2;
  double2* Q = G + 3 * kk2;
  double2* Ht = G + 4 * kk2;
  double2* Ga = G + c0 + (size_t)c0 * k;  // G_aa -> R (scaled Cholesky factor)
  double2* Ha = H + c0 + (size_t)c0 * k;  // H_aa
  double* dinv = dwork + d.kv * 4;  // 4 k-length scratch vectors per problem
  double* lam = dinv + k;
  int* perm = reinterpret_cast<int*>(lam + k);
  double* th = theta + d.kv;
  __shared__ int s_flag;
  __shared__ double s_red[32];
  const int nn = n * n;

  // (0) projection against the locked block: with G_la = V_l^H W_a and
  // H_la = V_l^H A W_a (Gram tiles of the locked rows), V_l^H V_l = I and
  // V_l^H A V_l = Theta_l,  W_a' = W_a - V_l G_la  has
  //   G' = G_aa - G_la^H G_la,
  //   H' = H_aa - G_la^H H_la - H_la^H G_la + G_la^H Theta_l G_la.
  if (c0 > 0) {
    for (int e = tid; e < nn; e += nt) {
      const int i = e % n, j = e / n;
      const double2* gi = G + (size_t)(c0 + i) * k;
      const double2* gj = G + (size_t)(c0 + j) * k;
      const double2* hi = H + (size_t)(c0 + i) * k;
      const double2* hj = H + (size_t)(c0 + j) * k;
      double2 sg = make_double2(0.0, 0.0), sh = make_double2(0.0, 0.0);
      for (int q = 0; q < c0; ++q) {
        const double2 a = gi[q], b = gj[q];
        cfmac(sg, a, b);                                 // conj(G_qi) G_qj
        cfmac(sh, a, hj[q]);                             // conj(G_qi) H_qj
        cfmac(sh, hi[q], b);                             // conj(H_qi) G_qj
        const double2 t = cmulc(a, b);
        sh = make_double2(sh.x - th[q] * t.x, sh.y - th[q] * t.y);  // - theta_q conj(G_qi) G_qj
      }
      double2& g = Ga[i + (size_t)j * k];
      double2& h = Ha[i + (size_t)j * k];
      g = csub(g, sg);
      h = csub(h, sh);
    }
    __syncthreads();
  }
  // (a) column scaling D = sqrt(diag G')
  for (int i = tid; i < n; i += nt) {
    const double g = Ga[i + (size_t)i * k].x;
    dinv[i] = g > 0.0 ? 1.0 / sqrt(g) : 1.0;
  }
  if (tid == 0) s_flag = 0;
  __syncthreads();
  for (int e = tid; e < nn; e += nt) {
    const int i = e % n, j = e / n;
    Ga[i + (size_t)j * k] = cscal(Ga[i + (size_t)j * k], dinv[i] * dinv[j]);
  }
  __syncthreads();
  // (b) Cholesky G' = R^H R, R upper, in place (right-looking)
  for (int q = 0; q < n; ++q) {
    if (tid == 0) {
      double piv = at(Ga, k, q, q).x;
      if (!(piv > 1e-28)) {
        piv = 1e-28;
        s_flag = 1;
      }
      at(Ga, k, q, q) = make_double2(sqrt(piv), 0.0);
    }
    __syncthreads();
    const double rinv = 1.0 / at(Ga, k, q, q).x;
    for (int j = q + 1 + tid; j < n; j += nt) at(Ga, k, q, j) = cscal(at(Ga, k, q, j), rinv);
    __syncthreads();
    const int m = n - q - 1;
    for (int e = tid; e < m * m; e += nt) {
      const int i = q + 1 + e / m, j = q + 1 + e % m;
      if (i <= j) {
        double2 v = at(Ga, k, i, j);
        const double2 a = at(Ga, k, q, i), b = at(Ga, k, q, j);
        // v -= conj(a) b
        v.x -= a.x * b.x + a.y * b.y;
        v.y -= a.x * b.y - a.y * b.x;
        at(Ga, k, i, j) = v;
      }
    }
    __syncthreads();
  }
  stamp(1);
  // (c) Minv = D^{-1} R^{-1} (upper triangular), column by column
  for (int e = tid; e < nn; e += nt) Mi[e % n + (size_t)(e / n) * k] = make_double2(0.0, 0.0);
  __syncthreads();
  for (int j = 0; j < n; ++j) {
    const double rjj = at(Ga, k, j, j).x;
    for (int i = tid; i <= j; i += nt) {
      double2 s = make_double2(i == j ? 1.0 : 0.0, 0.0);
      for (int q = i; q < j; ++q) {
        // s -= Rinv(i,q) R(q,j)
        const double2 a = at(Mi, k, i, q), b = at(Ga, k, q, j);
        s.x -= a.x * b.x - a.y * b.y;
        s.y -= a.x * b.y + a.y * b.x;
      }
      at(Mi, k, i, j) = cscal(s, 1.0 / rjj);
    }
    __syncthreads();
  }
  for (int e = tid; e < nn; e += nt) {
    const int i = e % n, j = e / n;
    Mi[i + (size_t)j * k] = cscal(Mi[i + (size_t)j * k], dinv[i]);
  }
  __syncthreads();
  stamp(2);
  // (d) T1 = H' Minv ; Ht = Minv^H T1 (Hermitian part)
  for (int e = tid; e < nn; e += nt) {
    const int i = e % n, j = e / n;
    double2 s = make_double2(0.0, 0.0);
    for (int q = 0; q <= j; ++q) cfma(s, at(Ha, k, i, q), at(Mi, k, q, j));
    Q[i + (size_t)j * k] = s;
  }
  __syncthreads();
  for (int e = tid; e < nn; e += nt) {
    const int i = e % n, j = e / n;
    double2 s = make_double2(0.0, 0.0);
    for (int q = 0; q <= i; ++q) cfmac(s, at(Mi, k, q, i), at(Q, k, q, j));
    Ht[i + (size_t)j * k] = s;
  }
  __syncthreads();
  for (int e = tid; e < nn; e += nt) {
    const int i = e % n, j = e / n;
    if (i < j) {
      const double2 a = at(Ht, k, i, j), b = at(Ht, k, j, i);
      const double2 h = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
      at(Ht, k, i, j) = h;
      at(Ht, k, j, i) = cconj(h);
    } else if (i == j) {
      at(Ht, k, i, i).y = 0.0;
    }
    Q[i + (size_t)j * k] = make_double2(i == j ? 1.0 : 0.0, 0.0);
  }
  __syncthreads();
  stamp(3);
  // (e) cyclic Jacobi in "position order": in every step position i is paired
  // with its mirror n-1-i, and after the rotations positions 1..n-1 shift by
  // one (round-robin tournament: every pair meets once in n-1 steps).  The
  // shift is folded into the update, which writes the rotated 2x2 blocks of
  // Ht (and the rotated column pairs of Q) to their new positions in a second
  // buffer, so each step is one read and one write of both matrices with
  // unit-stride warp accesses.  Ht ping-pongs with the H storage, Q with the
  // active block of the G storage (the Cholesky factor, no longer needed);
  // Q's rows stay in the basis order and its columns follow Ht's diagonal,
  // which is all the sort below needs.
  __shared__ double s_c[256], s_s[256];
  __shared__ double2 s_e[256];
  const int half = n / 2;
  double2* hc = Ht;  // current Ht
  double2* hn = H;   // next Ht
  double2* qc = Q;
  double2* qn = Ga;
  auto shift = [&](int pos) { return pos == 0 ? 0 : (pos == n - 1 ? 1 : pos + 1); };
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    double off = 0.0, dia = 0.0;
    for (int e = tid; e < nn; e += nt) {
      const int i = e % n, j = e / n;
      const double2 v = hc[i + (size_t)j * k];
      if (i != j) off += v.x * v.x + v.y * v.y;
      else dia += v.x * v.x;
    }
    for (int o = 16; o > 0; o >>= 1) {
      off += __shfl_xor_sync(0xffffffffu, off, o);
      dia += __shfl_xor_sync(0xffffffffu, dia, o);
    }
    __shared__ double s_off[32], s_dia[32];
    if ((tid & 31) == 0) {
      s_off[tid >> 5] = off;
      s_dia[tid >> 5] = dia;
    }
    __syncthreads();
    if (tid == 0) {
      double a = 0.0, b = 0.0;
      for (int w = 0; w < (nt >> 5); ++w) {
        a += s_off[w];
        b += s_dia[w];
      }
      s_red[0] = a;
      s_red[1] = b;
    }
    __syncthreads();
    // |off| <= 3e-14 |diag|: with eigenvalue gaps >= 1e-3 lambda_max this
    // leaves eigenvector errors below 1e-10, far under the residual target
    if (s_red[0] <= 1e-27 * s_red[1]) break;
    for (int step = 0; step < n - 1; ++step) {
      // rotation of pair r = (r, n-1-r): J (p,p)=c (p,q)=s (q,p)=-s e (q,q)=c e, e = e^{-i phi}
      for (int r = tid; r < half; r += nt) {
        const int pa = r, qb = n - 1 - r;
        const double2 g = at(hc, k, pa, qb);
        const double rr = hypot(g.x, g.y);
        const double app = at(hc, k, pa, pa).x, aqq = at(hc, k, qb, qb).x;
        double c = 1.0, s = 0.0;
        double2 em = make_double2(1.0, 0.0);
        if (rr > 1e-300 && rr > 1e-18 * sqrt(fabs(app * aqq))) {
          em = make_double2(g.x / rr, -g.y / rr);
          const double tau = (aqq - app) / (2.0 * rr);
          const double tt = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
          c = 1.0 / sqrt(1.0 + tt * tt);
          s = tt * c;
        }
        s_c[r] = c;
        s_s[r] = s;
        s_e[r] = em;
      }
      __syncthreads();
      // Ht <- J^H Ht J on every 2x2 block (rows r', n-1-r'; columns r, n-1-r), shifted
      for (int e = tid; e < half * half; e += nt) {
        const int r = e / half, rp = e - r * half;
        const int p = r, q = n - 1 - r, pp = rp, qq = n - 1 - rp;
        const double c = s_c[r], s = s_s[r];
        const double2 em = s_e[r];
        const double c2 = s_c[rp], s2 = s_s[rp];
        const double2 ep = cconj(s_e[rp]);
        const double2 a_pp = at(hc, k, pp, p), a_qp = at(hc, k, qq, p);
        const double2 a_pq = at(hc, k, pp, q), a_qq = at(hc, k, qq, q);
        // columns: X = A J
        const double2 t1 = cmul(a_pq, em), t2 = cmul(a_qq, em);
        const double2 x_pp = make_double2(c * a_pp.x - s * t1.x, c * a_pp.y - s * t1.y);
        const double2 x_qp = make_double2(c * a_qp.x - s * t2.x, c * a_qp.y - s * t2.y);
        const double2 x_pq = make_double2(s * a_pp.x + c * t1.x, s * a_pp.y + c * t1.y);
        const double2 x_qq = make_double2(s * a_qp.x + c * t2.x, s * a_qp.y + c * t2.y);
        // rows: B = J'^H X, J'^H (p',p')=c' (p',q')=-s' conj(e') (q',p')=s' (q',q')=c' conj(e')
        const double2 u1 = cmul(x_qp, ep), u2 = cmul(x_qq, ep);
        double2 b_pp = make_double2(c2 * x_pp.x - s2 * u1.x, c2 * x_pp.y - s2 * u1.y);
        double2 b_qp = make_double2(s2 * x_pp.x + c2 * u1.x, s2 * x_pp.y + c2 * u1.y);
        double2 b_pq = make_double2(c2 * x_pq.x - s2 * u2.x, c2 * x_pq.y - s2 * u2.y);
        double2 b_qq = make_double2(s2 * x_pq.x + c2 * u2.x, s2 * x_pq.y + c2 * u2.y);
        if (rp == r) {
          // diagonal block: the rotated pair is decoupled exactly
          if (s != 0.0) b_pq = b_qp = make_double2(0.0, 0.0);
          b_pp.y = 0.0;
          b_qq.y = 0.0;
        }
        const int np_ = shift(p), nq_ = shift(q), npp = shift(pp), nqq = shift(qq);
        at(hn, k, npp, np_) = b_pp;
        at(hn, k, nqq, np_) = b_qp;
        at(hn, k, npp, nq_) = b_pq;
        at(hn, k, nqq, nq_) = b_qq;
      }
      // Q <- Q J, columns shifted
      for (int e = tid; e < half * n; e += nt) {
        const int r = e / n, i = e - r * n;
        const int p = r, q = n - 1 - r;
        const double c = s_c[r], s = s_s[r];
        const double2 em = s_e[r];
        const double2 qp = at(qc, k, i, p), qq = cmul(at(qc, k, i, q), em);
        at(qn, k, i, shift(p)) = make_double2(c * qp.x - s * qq.x, c * qp.y - s * qq.y);
        at(qn, k, i, shift(q)) = make_double2(s * qp.x + c * qq.x, s * qp.y + c * qq.y);
      }
      __syncthreads();
      double2* t = hc;
      hc = hn;
      hn = t;
      t = qc;
      qc = qn;
      qn = t;
    }
  }
  if (qc != Q) {
    // bring Q home: its other buffer is written below
    for (int e = tid; e < nn; e += nt) {
      const size_t o = e % n + (size_t)(e / n) * k;
      Q[o] = qc[o];
    }
    __syncthreads();
  }
  stamp(4);
  // (f) sort ascending (rank sort, ties by index)
  for (int i = tid; i < n; i += nt) lam[i] = at(hc, k, i, i).x;
  __syncthreads();
  for (int i = tid; i < n; i += nt) {
    const double li = lam[i];
    int r = 0;
    for (int j = 0; j < n; ++j) {
      const double lj = lam[j];
      r += (lj < li) || (lj == li && j < i);
    }
    perm[r] = i;
  }
  __syncthreads();
  for (int r = tid; r < n; r += nt) th[c0 + r] = lam[perm[r]];
  // (g) C_a = Minv Q[:, perm]; the rotation's coefficients of the active
  // columns over the whole block are [-G_la C_a ; C_a] (the V_l part undoes
  // the projection), stored in columns c0.. of the G storage
  double2* T = c0 > 0 ? H : Ga;  // C_a (H is free after the sort)
  for (int e = tid; e < nn; e += nt) {
    const int i = e % n, j = e / n;
    const int pj = perm[j];
    double2 s = make_double2(0.0, 0.0);
    for (int q = i; q < n; ++q) cfma(s, at(Mi, k, i, q), at(Q, k, q, pj));
    T[i + (size_t)j * k] = s;
  }
  __syncthreads();
  if (c0 > 0) {
    // X = -G_la C_a into Ht (free), then both parts into G's columns c0..
    for (int e = tid; e < c0 * n; e += nt) {
      const int q = e % c0, j = e / c0;
      double2 s = make_double2(0.0, 0.0);
      for (int i = 0; i < n; ++i) cfma(s, G[q + (size_t)(c0 + i) * k], T[i + (size_t)j * k]);
      Ht[q + (size_t)j * k] = make_double2(-s.x, -s.y);
    }
    __syncthreads();
    for (int e = tid; e < k * n; e += nt) {
      const int row = e % k, j = e / k;
      G[row + (size_t)(c0 + j) * k] = row < c0 ? Ht[row + (size_t)j * k] : T[(row - c0) + (size_t)j * k];
    }
    __syncthreads();
  }
  stamp(5);
  // (h) next window [lam_cut, lam_max] and Chebyshev coefficients
  if (tid == 0) {
    ProbState& S = ps[p];
    double cut = th[k - 1];
    if (fixed_cut || (first_iter && S.lam_cut > 0.0)) cut = S.lam_cut;
    if (cut >= S.lam_max - 1e-3) cut = S.lam_max - 1e-3;
    if (cut < 1e-6) cut = 1e-6;
    S.lam_cut = cut;
    const double al = 2.0 / (S.lam_max - cut);
    S.c_hop = al;
    S.c_diag = (S.lam_max + cut - 12.0) / (S.lam_max - cut);
    S.chol_fail = s_flag;
    S.theta_min = th[0];
  }
  stamp(6);
}

// ------------------------------------------------- Chebyshev coefficients --
// Scaled recurrence for a filter of degree m (chosen by the host each
// iteration).  With E_1 = S/2, E_0 = 0 and
//   E_{n+1} = 2B E_n - E_{n-1} + T_n(theta_B) S,
// T_m(B) V = V T_m(Theta_B) + E_m exactly (S = 2(BV - V Theta_B)).  Each
// column is carried as E'_n = E_n / nu_n, nu_n = max(1, |T_n|), so every FP32
// value stays O(|S|):
//   step 1: E'_2 = (B S + T_1 S) / nu_2
//   step 2: E'_3 = (2 nu_2 B E'_2 + (T_2 - 1/2) S) / nu_3
//   step n: E'_{n+1} = (2 nu_n B E'_n - nu_{n-1} E'_{n-1} + T_n S) / nu_{n+1}
//   final : W' = (T_m / nu_m) V + E'_m   (= W / nu_m)
// A direct pass (ProbState::direct) filters V itself: S holds V in FP32
// (k_direct_start) and X_n = T_n(B) V, carried as X'_n = X_n / nu_n:
//   step 1: X'_1 = B S / nu_1
//   step 2: X'_2 = (2 nu_1 B X'_1 - S) / nu_2
//   step n: X'_n = (2 nu_{n-1} B X'_{n-1} - nu_{n-2} X'_{n-2}) / nu_n   (no S)
//   final : W' = X'_{m-1}   (T_m / nu_m = 0: the pass applies T_{m-1}(B))
__global__ void k_coef(const ProbDesc* __restrict__ pd, const ProbState* __restrict__ ps, int np,
                       const double* __restrict__ theta, double* __restrict__ tcoef, double* __restrict__ scol, int m,
                       const int* __restrict__ dm) {
  if (dm) m = *dm;  // degree decided on the device (the device-side loop)
  const int p = blockIdx.x;
  if (p >= np || !ps[p].active) return;
  const ProbDesc d = pd[p];
  const ProbState S = ps[p];
  const int k = d.k;
  const double* th = theta + d.kv;
  double* tc = tcoef + d.tc;
  for (int j = threadIdx.x; j < k; j += blockDim.x) {
    const double tb = 1.0 + 2.0 * (S.lam_cut - th[j]) / (S.lam_max - S.lam_cut);
    double tn[kMaxFilterDeg + 2], nu[kMaxFilterDeg + 2];
    tn[0] = 1.0;
    tn[1] = tb;
    for (int n = 2; n <= m; ++n) tn[n] = 2.0 * tb * tn[n - 1] - tn[n - 2];
    for (int n = 0; n <= m; ++n) nu[n] = fmax(1.0, fabs(tn[n]));
    if (S.direct) {
      for (int n = 1; n < m; ++n) {
        const double a = n == 1 ? 1.0 / nu[1] : 2.0 * nu[n - 1] / nu[n];
        const double z = n >= 3 ? -nu[n - 2] / nu[n] : 0.0;
        const double g = n == 2 ? -1.0 / nu[2] : 0.0;
        tc[((size_t)n * 3 + 0) * k + j] = a;
        tc[((size_t)n * 3 + 1) * k + j] = z;
        tc[((size_t)n * 3 + 2) * k + j] = g;
      }
      tc[((size_t)m * 3 + 0) * k + j] = 0.0;
      scol[d.kv + j] = -2.0 * S.c_hop;
      continue;
    }
    for (int n = 1; n < m; ++n) {
      double a, z, g;
      if (n == 1) {
        a = 1.0 / nu[2];
        z = 0.0;
        g = tn[1] / nu[2];
      } else if (n == 2) {
        a = 2.0 * nu[2] / nu[3];
        z = 0.0;
        g = (tn[2] - 0.5) / nu[3];
      } else {
        a = 2.0 * nu[n] / nu[n + 1];
        z = -nu[n - 1] / nu[n + 1];
        g = tn[n] / nu[n + 1];
      }
      tc[((size_t)n * 3 + 0) * k + j] = a;
      tc[((size_t)n * 3 + 1) * k + j] = z;
      tc[((size_t)n * 3 + 2) * k + j] = g;
    }
    tc[((size_t)m * 3 + 0) * k + j] = tn[m] / nu[m];
    scol[d.kv + j] = -2.0 * S.c_hop;
  }
}

// ---------------------------------------------------------------- rotate ---
constexpr int RR = 128, RC = 32, RK = 8, RS = 3;
constexpr int kRotStage = RK * RR + RK * RC;  // double2 per stage
constexpr int kRotSmem = RS * kRotStage * (int)sizeof(double2);

// V = W C on the FP64 tensor path (mma.sync m8n8k4 f64): CTA tile 128 rows x
// 32 columns, W and C slabs of RK columns/rows through a three-stage cp.async
// ring (dynamic shared memory), each warp a 32 x 32 sub-tile of 4 x 4 8x8 MMA
// tiles; the complex product as four real MMAs (Vr += Wr Cr - Wi Ci,
// Vi += Wr Ci + Wi Cr).  Against the same tile on the FP64 FMA pipe (8 x 4
// complex per thread, 246 registers): +7% for the dense phase.
__global__ void __launch_bounds__(128) k_rotate(const ProbDesc* __restrict__ pd, const ProbState* __restrict__ ps,
                                                     const int* __restrict__ start, int np,
                                                     const double2* __restrict__ Wp, const double2* __restrict__ KK,
                                                     double2* __restrict__ Vp) {
  const int p = find_prob(start, np, blockIdx.x);
  if (!ps[p].active) return;
  const ProbDesc d = pd[p];
  const int nct = d.k / RC;
  const int t = blockIdx.x - start[p];
  const int rt = t / nct, ct = t - rt * nct;
  const int row0 = rt * RR, col0 = ct * RC;
  if (col0 < ps[p].c0) return;  // frozen columns keep their Ritz vectors
  const int k = d.k;
  const double2* C = KK + d.kk;
  const double2* Wb = Wp + d.blk;
  extern __shared__ double2 rsm[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wr0 = warp * 32;             // warp's rows within the CTA tile
  const int fr = lane >> 2, fk = lane & 3;  // fragment row / k index
  double accr[4][4][2], acci[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) accr[i][j][0] = accr[i][j][1] = acci[i][j][0] = acci[i][j][1] = 0.0;
  auto load = [&](int q0, int b) {
    double2* sW = rsm + b * kRotStage;
    double2* sC = sW + RK * RR;
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int idx = threadIdx.x + 128 * e;
      const int c = idx >> 7, r = idx & 127;
      const int row = row0 + r;
      const bool ok = row < d.dim;
      cp_async16(sW + c * RR + r, Wb + (size_t)LAPH_IX(q0 + c, k) * d.dim + (ok ? row : 0), ok);
    }
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int idx = threadIdx.x + 128 * e;
      const int c = idx & 31, r = idx >> 5;
      cp_async16(sC + r * RC + c, C + (size_t)LAPH_IX(col0 + c, k) * k + LAPH_IX(q0 + r, k), true);
    }
    cp_async_commit();
  };
  const int nstep = k / RK;
#pragma unroll
  for (int s = 0; s < RS - 1; ++s) {
    if (s < nstep) load(s * RK, s);
    else cp_async_commit();
  }
  for (int it = 0; it < nstep; ++it) {
    cp_async_wait<RS - 2>();
    __syncthreads();
    if (it + RS - 1 < nstep) load((it + RS - 1) * RK, (it + RS - 1) % RS);
    else cp_async_commit();
    const double2* sW = rsm + (it % RS) * kRotStage;
    const double2* sC = sW + RK * RR;
#pragma unroll
    for (int ks = 0; ks < RK / 4; ++ks) {
      const int q = ks * 4 + fk;
      double ar[4], ai[4], br[4], bi[4], bn[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const double2 a = sW[q * RR + wr0 + 8 * i + fr];  // A(row fr, k fk) of row tile i
        ar[i] = a.x;
        ai[i] = a.y;
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const double2 b = sC[q * RC + 8 * j + fr];  // B(k fk, col fr) of column tile j
        br[j] = b.x;
        bi[j] = b.y;
        bn[j] = -b.y;
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma884(accr[i][j], ar[i], br[j]);
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma884(acci[i][j], ar[i], bi[j]);
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma884(accr[i][j], ai[i], bn[j]);
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma884(acci[i][j], ai[i], br[j]);
    }
  }
  cp_async_wait<0>();
  // D(row fr, cols 2 fk, 2 fk + 1) of each 8x8 tile
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int row = row0 + wr0 + 8 * i + fr;
    if (row >= d.dim) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int col = col0 + 8 * j + 2 * fk + e;
        Vp[(size_t)d.blk + (size_t)col * d.dim + row] = make_double2(accr[i][j][e], acci[i][j][e]);
      }
  }
}

// R = A V - V Theta in FP64 (A = -Delta), S = -2 c_hop R in FP32 for the next
// filter, and per-CTA partial sums of |R_j|^2.  One thread per (site,
// column); CTA = 128 sites of one column.
__global__ void __launch_bounds__(128) k_residual64(const ProbDesc* __restrict__ pd, const ProbState* __restrict__ ps,
                                                    const int* __restrict__ start, int np,
                                                    const double2* __restrict__ U64, const double2* __restrict__ Vp,
                                                    const double* __restrict__ theta, float2* __restrict__ Sp,
                                                    double* __restrict__ rpart) {
  const int p = find_prob(start, np, blockIdx.x);
  if (!ps[p].active) return;
  const ProbDesc d = pd[p];
  const int nst = (d.V3 + 127) >> 7;
  const int t = blockIdx.x - start[p];
  const int st = t % nst, j = t / nst;
  if (j < ps[p].c0) return;  // frozen column: its residual partials stand
  const int s = st * 128 + threadIdx.x;
  double rr = 0.0;
  if (s < d.V3) {
    const Lat g{d.L, d.L * d.L, d.V3};
    const double2* U = U64 + d.u64;
    const size_t col = (size_t)d.blk + (size_t)j * d.dim;
    const double2* x = Vp + col;
    int sx, sy, sz;
    site_xyz(g, s, sx, sy, sz);
    double2 acc[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
#pragma unroll
    for (int mu = 0; mu < 3; ++mu) {
      const int u = nb_up(g, sx, sy, sz, mu), dn = nb_dn(g, sx, sy, sz, mu);
      double2 xu[3], xd[3];
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        xu[b] = __ldg(x + (size_t)b * d.V3 + u);
        xd[b] = __ldg(x + (size_t)b * d.V3 + dn);
      }
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          cfma(acc[a], __ldg(U + (size_t)(mu * 9 + 3 * a + b) * d.V3 + s), xu[b]);
          cfmac(acc[a], __ldg(U + (size_t)(mu * 9 + 3 * b + a) * d.V3 + dn), xd[b]);
        }
    }
    const double th = __ldg(theta + d.kv + j);
    const double sc = -2.0 * ps[p].c_hop;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double2 xs = __ldg(x + (size_t)a * d.V3 + s);
      const double2 r = make_double2((6.0 - th) * xs.x - acc[a].x, (6.0 - th) * xs.y - acc[a].y);
      rr += r.x * r.x + r.y * r.y;
      Sp[col + (size_t)a * d.V3 + s] = make_float2((float)(sc * r.x), (float)(sc * r.y));  // colour-major
    }
  }
  // block reduction (fixed order)
  for (int o = 16; o > 0; o >>= 1) rr += __shfl_xor_sync(0xffffffffu, rr, o);
  __shared__ double red[4];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = rr;
  __syncthreads();
  if (threadIdx.x == 0) rpart[d.rp + (size_t)st * d.k + j] = red[0] + red[1] + red[2] + red[3];
}

// The same residual laid out like the FP64 block stencil A W: CTA = 128 sites x
// a block of kColsFP64 columns, the site's forward links in registers and its
// backward links in shared memory, read once per column block instead of
// once per (site, column).  Each thread leaves |r|^2 of its site and column in
// shared memory (FP32: one site's share of a norm needs no more); after the
// column loop the CTA reduces the 128 sites of every column in a fixed order
// (FP64 sums) into the same per-tile partials as the kernel above, so the
// column loop carries no per-column reduction.
constexpr int kResidSmem = kStencil64Smem + kColsFP64 * kSites64 * (int)sizeof(float);

__global__ void __launch_bounds__(kSites64, 3)
    k_residual64_cols(const ProbDesc* __restrict__ pd, const ProbState* __restrict__ ps, const int* __restrict__ start,
                      int np, const double2* __restrict__ U64, const double2* __restrict__ Vp,
                      const double* __restrict__ theta, float2* __restrict__ Sp, double* __restrict__ rpart) {
  const int p = find_prob(start, np, blockIdx.x);
  if (!ps[p].active) return;
  const ProbDesc d = pd[p];
  const int nst = (d.V3 + kSites64 - 1) / kSites64;
  const int t = blockIdx.x - start[p];
  const int st = t % nst, cb = t / nst;
  const int c0 = ps[p].c0;
  const int j0 = cb * kColsFP64, j1 = min(d.k, j0 + kColsFP64);
  if (j1 <= c0) return;  // frozen columns: their residual partials stand
  const int jstart = max(j0, c0);
  // threads past the last site compute the last site again and write nothing
  const bool valid = st * kSites64 + (int)threadIdx.x < d.V3;
  const int s = min(st * kSites64 + (int)threadIdx.x, d.V3 - 1);
  extern __shared__ double2 s64[];
  double2 (*sUb)[kSites64] = reinterpret_cast<double2 (*)[kSites64]>(s64);
  float (*sPart)[kSites64] = reinterpret_cast<float (*)[kSites64]>(s64 + 27 * kSites64);
  const Lat g{d.L, d.L * d.L, d.V3};
  int up[3], dn[3], sx, sy, sz;
  site_xyz(g, s, sx, sy, sz);
#pragma unroll
  for (int mu = 0; mu < 3; ++mu) {
    up[mu] = nb_up(g, sx, sy, sz, mu);
    dn[mu] = nb_dn(g, sx, sy, sz, mu);
  }
  Links64 l;
  load_links64(U64 + d.u64, g, s, dn, l, sUb);
  const double sc = -2.0 * ps[p].c_hop;
#pragma unroll 1
  for (int j = jstart; j < j1; ++j) {
    const size_t col = (size_t)d.blk + (size_t)j * d.dim;
    const double2* x = Vp + col;
    double2 acc[3];
    hop64_col(l, sUb, d.V3, up, dn, x, acc);
    const double th = __ldg(theta + d.kv + LAPH_IX(j, d.k));
    double r2 = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double2 xs = __ldg(x + (size_t)a * d.V3 + s);
      const double2 r = make_double2((6.0 - th) * xs.x - acc[a].x, (6.0 - th) * xs.y - acc[a].y);
      r2 += r.x * r.x + r.y * r.y;
      if (valid) Sp[col + (size_t)a * d.V3 + s] = make_float2((float)(sc * r.x), (float)(sc * r.y));
    }
    sPart[LAPH_IX(j - j0, kColsFP64)][threadIdx.x] = valid ? (float)r2 : 0.f;
  }
  __syncthreads();
  // column c = tid / 4 summed by 4 threads over 32 sites each, then across them
  const int c = threadIdx.x >> 2, q = threadIdx.x & 3;
  double sum = 0.0;
  if (j0 + c >= jstart && j0 + c < j1)
#pragma unroll 8
    for (int i = 0; i < kSites64 / 4; ++i) sum += (double)sPart[c][q * (kSites64 / 4) + i];
  sum += __shfl_xor_sync(0xffffffffu, sum, 1);
  sum += __shfl_xor_sync(0xffffffffu, sum, 2);
  if (q == 0 && j0 + c >= jstart && j0 + c < j1) rpart[d.rp + (size_t)st * d.k + j0 + c] = sum;
}

// ------------------------------------------------------- residuals/conv ----
__global__ void k_resid(const ProbDesc* __restrict__ pd, ProbState* __restrict__ ps, const double* __restrict__ rpart,
                        double* __restrict__ resid, double tol, int* __restrict__ n_active) {
  const int p = blockIdx.x;
  if (!ps[p].active) return;
  const ProbDesc d = pd[p];
  __shared__ double s_max[32];
  __shared__ int s_cnt[32];
  double mx = 0.0;
  int cnt = 0;
  const double lmax = ps[p].lam_max;
  for (int j = threadIdx.x; j < d.k; j += blockDim.x) {
    double s = 0.0;
    for (int r = 0; r < d.nrt; ++r) s += rpart[d.rp + (size_t)r * d.k + j];
    const double rr = sqrt(s) / lmax;
    resid[d.kv + j] = rr;
    if (j < d.nev) {
      mx = fmax(mx, rr);
      cnt += rr <= tol;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  }
  if ((threadIdx.x & 31) == 0) {
    s_max[threadIdx.x >> 5] = mx;
    s_cnt[threadIdx.x >> 5] = cnt;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    int c = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      m = fmax(m, s_max[w]);
      c += s_cnt[w];
    }
    ProbState& S = ps[p];
    S.max_resid = m;
    S.nconv = c;
    S.iters += 1;
    // lock the leading columns whose residual is well below tol: the filter
    // leaves them as they are (W_j = V_j); they stay in every Rayleigh-Ritz
    // and are re-measured, so one that drifts up is unlocked next iteration
    int nl = 0;
    while (nl < d.nev && resid[d.kv + nl] <= 0.3 * tol) ++nl;
    S.nlock = nl;
    // frozen block for the Rayleigh-Ritz: whole Gram tiles of locked columns,
    // never shrinking (a frozen column is not re-measured, so it stays locked)
    S.c0 = max(S.c0, min(nl / GT * GT, d.k - GT));
    if (c >= d.nev) S.active = 0;
    else atomicAdd(n_active, 1);
  }
}

// ---------------------------------------------------------------- output ---
// fix_phase (modules/eigensystem.cpp:4-30) on V[:, :nev]: phase_j = arg V(0,j),
// V_j <- e^{-i phase_j} V_j; also |V_j|^2 for tr(V^dag V).  One CTA per column.
__global__ void k_phase_fix(const ProbDesc* __restrict__ pd, const int* __restrict__ start, int np,
                            double2* __restrict__ Vp, double* __restrict__ phases, double* __restrict__ norms,
                            int apply) {
  const int p = find_prob(start, np, blockIdx.x);
  const ProbDesc d = pd[p];
  const int j = blockIdx.x - start[p];
  if (j >= d.nev) return;
  double2* v = Vp + d.blk + (size_t)j * d.dim;
  const double2 v0 = v[0];
  const double ph = atan2(v0.y, v0.x);
  double sn, cs;
  sincos(ph, &sn, &cs);
  const double2 f = apply ? make_double2(cs, -sn) : make_double2(1.0, 0.0);
  double nrm = 0.0;
  __syncthreads();
  for (int i = threadIdx.x; i < d.dim; i += blockDim.x) {
    const double2 x = v[i];
    nrm += x.x * x.x + x.y * x.y;
    if (apply) v[i] = cmul(f, x);
  }
  __shared__ double red[256];
  red[threadIdx.x] = nrm;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    phases[d.kv + j] = ph;
    norms[d.kv + j] = red[0];
  }
}

// ---------------------------------------------------------- start window --
// State of a random start block used without a first Rayleigh-Ritz (window
// from the learned model or fixed): every column gets the Ritz value lam_max,
// where T_n(theta_B) = (-1)^n, so the first filter pass runs entirely through
// the FP32 correction E = T_m(B) V - V T_m(theta_B) (accurate to FP32, which
// is all a first pass needs); the window is the one already in the state.
__global__ void k_start_window(const ProbDesc* __restrict__ pd, ProbState* __restrict__ ps, int np,
                               double* __restrict__ theta) {
  const int p = blockIdx.x;
  if (p >= np) return;
  const ProbDesc d = pd[p];
  ProbState& S = ps[p];
  for (int j = threadIdx.x; j < d.k; j += blockDim.x) theta[d.kv + j] = S.lam_max;
  if (threadIdx.x == 0) {
    double cut = S.lam_cut;
    if (cut >= S.lam_max - 1e-3) cut = S.lam_max - 1e-3;
    if (cut < 1e-6) cut = 1e-6;
    S.lam_cut = cut;
    S.c_hop = 2.0 / (S.lam_max - cut);
    S.c_diag = (S.lam_max + cut - 12.0) / (S.lam_max - cut);
    S.chol_fail = 0;
    S.theta_min = S.lam_max;
  }
}

// --------------------------------------------------------------- output ---
// Colour-major columns (c*V3 + site) -> the reference's 3*site + colour order.
__global__ void k_to_reference(const double2* __restrict__ in, double2* __restrict__ out, int V3, int nev) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= V3) return;
  const size_t col = (size_t)blockIdx.y * 3 * V3;
#pragma unroll
  for (int c = 0; c < 3; ++c) out[col + 3 * (size_t)s + c] = __ldg(in + col + (size_t)c * V3 + s);
}

// ------------------------------------------------------------- launchers ---
int start_window(const ProbDesc* pd, ProbState* ps, int np, double* theta, cudaStream_t st) {
  k_start_window<<<np, 256, 0, st>>>(pd, ps, np, theta);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}
int to_reference(const double2* in, double2* out, int V3, int nev, cudaStream_t st) {
  k_to_reference<<<dim3((V3 + 255) / 256, nev), 256, 0, st>>>(in, out, V3, nev);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}
int dense_init() {
  LAPH_CUDA_TRY(cudaFuncSetAttribute(k_gram, cudaFuncAttributeMaxDynamicSharedMemorySize, kGramSmem));
  LAPH_CUDA_TRY(cudaFuncSetAttribute(k_rotate, cudaFuncAttributeMaxDynamicSharedMemorySize, kRotSmem));
  LAPH_CUDA_TRY(cudaFuncSetAttribute(k_residual64_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, kResidSmem));
  LAPH_TRY(neglap64_init());
  return LAPH_OK;
}
int gram(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, int chunk_rows,
         const double2* W, const double2* Y, double2* gpart, cudaStream_t st) {
  k_gram<<<nblk, 64, kGramSmem, st>>>(pd, ps, start, np, chunk_rows, W, Y, gpart);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}
int gram_reduce(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, const double2* gpart,
                double2* KK, cudaStream_t st) {
  k_gram_reduce<<<nblk, 256, 0, st>>>(pd, ps, start, np, gpart, KK);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}
int small_dense(const ProbDesc* pd, ProbState* ps, int np, double2* KK, double* theta, double* tcoef, double* scol,
                double* dwork, int first_iter, int fixed_cut, int max_sweeps, unsigned long long* tstamp,
                cudaStream_t st) {
  k_small<<<np, 1024, 0, st>>>(pd, ps, KK, theta, tcoef, scol, dwork, first_iter, fixed_cut, max_sweeps, tstamp);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}
int coef(const ProbDesc* pd, const ProbState* ps, int np, const double* theta, double* tcoef, double* scol, int m,
         const int* dm, cudaStream_t st) {
  k_coef<<<np, 256, 0, st>>>(pd, ps, np, theta, tcoef, scol, m, dm);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}
int rotate(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, const double2* W,
           const double2* KK, double2* V, cudaStream_t st) {
  k_rotate<<<nblk, 128, kRotSmem, st>>>(pd, ps, start, np, W, KK, V);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}
int residual64(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, const double2* U64,
               const double2* V, const double* theta, float2* S, double* rpart, cudaStream_t st) {
  k_residual64<<<nblk, 128, 0, st>>>(pd, ps, start, np, U64, V, theta, S, rpart);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}
int residual64_cols(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, const double2* U64,
                    const double2* V, const double* theta, float2* S, double* rpart, cudaStream_t st) {
  k_residual64_cols<<<nblk, kSites64, kResidSmem, st>>>(pd, ps, start, np, U64, V, theta, S, rpart);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}
int resid_check(const ProbDesc* pd, ProbState* ps, int np, const double* rpart, double* resid, double tol,
                int* n_active, cudaStream_t st) {
  k_resid<<<np, 256, 0, st>>>(pd, ps, rpart, resid, tol, n_active);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}
int phase_fix(const ProbDesc* pd, const int* start, int np, int nblk, double2* V, double* phases, double* norms,
              int apply, cudaStream_t st) {
  k_phase_fix<<<nblk, 256, 0, st>>>(pd, start, np, V, phases, norms, apply);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}

}  // namespace laph
