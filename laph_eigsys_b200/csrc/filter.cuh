// filter.cuh -- launchers of the block stencils (filter.cu).
#pragma once
#include "batch.cuh"

namespace laph {
// FP64 links -> FP32 or BF16 (+ per-site scale) filter links; nblk blocks of 128 sites.
int pack_links(const ProbDesc* pd, const int* start, int np, int nblk, const double2* U64, float2* Uf32, void* Ubf,
               float* scale, int bf16, cudaStream_t st);
// One Chebyshev step Y_j = a_j (c_hop hop(X_j) + c_diag X_j) + z_j Z_j + g_j S_j (FP32)
// with (a, z, g) = tcoef[step][0..2][j]; final_step writes W_j = tcoef[step+1][0][j] V_j + Y_j
// in FP64 instead of Y.  variant 0: per-thread FP64 coefficients; 1: FP32 coefficients
// staged in shared memory, backward links in shared memory; 2: as 1 with the backward
// links in tensor memory; 3: as 2 with every vector operand staged in shared memory by a
// bulk-copy pipeline (needs tile 128 and cheb_staged_ok(L) for every problem; lmax = the
// largest L of the batch; a pipeline wait that gives up sets *err); 4: as 2 on 512-site
// bricks (TX = 128 / L planes x 4 z-rows; tile 512, same L condition); 5: as 2 with each
// thread's next-column operands in flight through cp.async.  Variants 1-5 need
// kb <= 64; larger blocks take variant 0.  tile: sites per CTA of variants 1 and 2 (64,
// 128 or 256; variant 0 uses 128); nblk must match it.  no_s: every active problem runs a
// direct pass, so a step past the second (Z present) has a zero S coefficient and variant 1
// skips reading S (the other variants read it and add 0).
int cheb_step(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, int kb, int bf16,
              const void* links, const float* scale, const float2* X, const float2* Z, const float2* S, float2* Y,
              const double2* V, double2* W, const double* tcoef, int step, bool final_step, int variant, int tile,
              int lmax, int* err, bool no_s, cudaStream_t st);
// Whether a lattice of extent L takes the staged variant (L even, L | 128, 128 | L^2, L <= 128).
bool cheb_staged_ok(int L);
// The start of a direct pass: S = FP32(V) for the unlocked columns of every active problem
// with ProbState::direct set (the filter's grid: nblk CTAs of tile sites x kb columns).
int direct_start(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, int kb, int tile,
                 const double2* V, float2* S, cudaStream_t st);
// Opt the filter's 256-site tile into its dynamic shared memory on the current device.
int cheb_init();
// Opt the FP64 stencil into its dynamic shared memory on the current device.
int neglap64_init();
// Y = (-Delta) W for every column, FP64.
int neglap64_batch(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, const double2* U64,
                   const double2* W, double2* Y, cudaStream_t st);
// Gaussian random start block.
int random_block(const ProbDesc* pd, const int* start, int np, int nblk, double2* W, uint64_t seed, cudaStream_t st);
}  // namespace laph
