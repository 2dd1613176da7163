// stencil64.cuh -- FP64 covariant-Laplacian stencil entry points (stencil64.cu).
#pragma once
#include "common.cuh"

namespace laph {
// State of the bounded grid barrier of the fused product (device memory,
// 16 bytes, one per stream that runs fused products).
struct GridBar {
  unsigned count, gen;
  int err, pad;
};
// Y[:,j] = c_hop*hop(X[:,j]) + c_diag*X[:,j] + c_z*Z[:,j] for j < ncol (Z may be null).
int hop64(const double2* U, int L, const double2* X, const double2* Z, double2* Y, size_t ld, int ncol, double c_hop,
          double c_diag, double c_z, cudaStream_t st);
// Y = T_deg(B) X; tmp holds 2*ld*ncol complex128.
int cheb64(const double2* U, int L, double lam_l, double lam_c, int deg, const double2* x, double2* y, double2* tmp,
           size_t ld, int ncol, cudaStream_t st);
// y = T_deg(B) x for ONE vector in one cooperative launch (falls back to hop64
// for deg <= 1); tmp holds 2*ld complex128; bar is this stream's barrier
// state.  bar->err becomes nonzero if a grid barrier gave up (it stays set
// until the caller clears it).  x must not overlap y or tmp.
int cheb64_fused(const double2* U, int L, double lam_l, double lam_c, int deg, const double2* x, double2* y,
                 double2* tmp, size_t ld, GridBar* bar, cudaStream_t st);
}  // namespace laph
