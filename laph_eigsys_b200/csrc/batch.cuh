// batch.cuh -- descriptors of a batch of timeslice eigenproblems that one
// kernel launch covers (possibly of different L and block width k), and the
// CTA -> problem lookup shared by every batched kernel.
#pragma once
#include "common.cuh"

namespace laph {
// Largest filter degree of a pass (laph_solve_opts.deg).
constexpr int kMaxFilterDeg = 128;


// One problem (timeslice).  All offsets are in elements of the pool they
// index.  Blocks of k vectors are column-major with column stride dim.
struct ProbDesc {
  int L, V3, dim, k, nev, mdeg;
  long long u64;   // FP64 links, site-minor [3][9][V3] (double2)
  long long uf;    // filter links [3][9][V3] (float2 or bf16x2)
  long long sc;    // per-site scale (float)
  long long blk;   // dim*k blocks (FP64 V, W, Y and FP32 S, E0..E2)
  long long kk;    // k*k matrices
  long long kv;    // per-column arrays (length k)
  long long gp;    // Gram partials
  long long rp;    // residual partials
  long long tc;    // Chebyshev coefficient table [(mdeg+1)][k]
  int nchunk;      // row chunks of the Gram reduction
  int nrt;         // row tiles of the rotation
};

// Window/state per problem, written by the device.
struct ProbState {
  double lam_cut, lam_max;   // Chebyshev window of this iteration
  double c_hop, c_diag;      // B = c_hop*hop + c_diag (maps [lam_cut, lam_max] -> [1, -1])
  double max_resid;          // max over wanted pairs of ||r|| / lam_max
  double theta_min;          // smallest Ritz value
  int active;                // 1 while iterating
  int nconv;                 // wanted pairs at tolerance
  int iters;                 // outer iterations done
  int chol_fail;             // Cholesky pivot clamped in the last iteration
  int nlock;                 // leading Ritz columns converged well below tol: not filtered
  int c0;                    // nlock rounded down to the Gram tile: columns [0, c0) are frozen
                             // (left out of the Rayleigh-Ritz, projected out of the rest)
  int direct;                // this pass filters V itself in FP32 (T_{m-1}(B) V), not the
                             // correction: set while the largest wanted residual is above
                             // laph_solve_opts.direct_resid
  int direct_off;            // a direct pass did not halve the residual: no more direct passes
  double resid_begin;        // max_resid when the current pass began
};

// Block index b -> problem p with start[p] <= b < start[p+1].
__device__ __forceinline__ int find_prob(const int* __restrict__ start, int np, int b) {
  int lo = 0, hi = np - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(start + mid) <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

}  // namespace laph
