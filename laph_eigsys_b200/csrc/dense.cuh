// dense.cuh -- launchers of the FP64 dense block operations (dense.cu).
#pragma once
#include "batch.cuh"

namespace laph {
constexpr int kGramTile = 32;   // block widths k are multiples of this
constexpr int kRotRows = 128;   // rows per rotation tile
// Opt the dense kernels into their dynamic shared memory on the current device.
int dense_init();
int gram(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, int chunk_rows,
         const double2* W, const double2* Y, double2* gpart, cudaStream_t st);
int gram_reduce(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, const double2* gpart,
                double2* KK, cudaStream_t st);
// Per problem: scaling, Cholesky, inverse, projected matrix, Jacobi, sort, C, next window.
// tstamp[p][0..kSmallPhases-1] receives the global timer (ns) at the phase boundaries.
constexpr int kSmallPhases = 7;
int small_dense(const ProbDesc* pd, ProbState* ps, int np, double2* KK, double* theta, double* tcoef, double* scol,
                double* dwork, int first_iter, int fixed_cut, int max_sweeps, unsigned long long* tstamp,
                cudaStream_t st);
// Chebyshev coefficient table and S scaling for a filter of degree m (or *dm
// when dm is not null: the degree the device-side loop chose).
int coef(const ProbDesc* pd, const ProbState* ps, int np, const double* theta, double* tcoef, double* scol, int m,
         const int* dm, cudaStream_t st);
int rotate(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, const double2* W,
           const double2* KK, double2* V, cudaStream_t st);
int residual64(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, const double2* U64,
               const double2* V, const double* theta, float2* S, double* rpart, cudaStream_t st);
// The same on CTAs of 128 sites x 32 columns (links read once per column block);
// nblk and start as for neglap64_batch.
int residual64_cols(const ProbDesc* pd, const ProbState* ps, const int* start, int np, int nblk, const double2* U64,
                    const double2* V, const double* theta, float2* S, double* rpart, cudaStream_t st);
int resid_check(const ProbDesc* pd, ProbState* ps, int np, const double* rpart, double* resid, double tol,
                int* n_active, cudaStream_t st);
// Ritz values lam_max and filter map of the state's window for a start block that
// skips the first Rayleigh-Ritz.
int start_window(const ProbDesc* pd, ProbState* ps, int np, double* theta, cudaStream_t st);
// nev colour-major columns of 3*V3 -> 3*site + colour order (out must not overlap in).
int to_reference(const double2* in, double2* out, int V3, int nev, cudaStream_t st);
int phase_fix(const ProbDesc* pd, const int* start, int np, int nblk, double2* V, double* phases, double* norms,
              int apply, cudaStream_t st);
}  // namespace laph
