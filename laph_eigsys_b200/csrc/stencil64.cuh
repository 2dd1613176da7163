// stencil64.cuh -- FP64 covariant-Laplacian stencil entry points (stencil64.cu).
#pragma once
#include "common.cuh"

namespace laph {
// State of the bounded grid barrier of the fused product (device memory,
// 16 bytes, zeroed once, one per stream that runs fused products): the
// arrival counter (bit 31 flips at every barrier) and the give-up flag.
struct GridBar {
  unsigned count, pad0;
  int err, pad1;
};
// Y[:,j] = c_hop*hop(X[:,j]) + c_diag*X[:,j] + c_z*Z[:,j] for j < ncol (Z may be null).
int hop64(const double2* U, int L, const double2* X, const double2* Z, double2* Y, size_t ld, int ncol, double c_hop,
          double c_diag, double c_z, cudaStream_t st);
// Y = T_deg(B) X; tmp holds 2*ld*ncol complex128.
int cheb64(const double2* U, int L, double lam_l, double lam_c, int deg, const double2* x, double2* y, double2* tmp,
           size_t ld, int ncol, cudaStream_t st);
// y = T_deg(B) x for ONE vector in one cooperative launch (falls back to hop64
// for deg <= 1); tmp holds 2*ld complex128; bar is this stream's barrier
// state.  If a grid barrier gives up, bar->err and *herr (a device-visible
// pointer to page-locked host memory) become 1; the caller then zeroes bar
// and *herr before the next launch.  x must not overlap y or tmp.
int cheb64_fused(const double2* U, int L, double lam_l, double lam_c, int deg, const double2* x, double2* y,
                 double2* tmp, size_t ld, GridBar* bar, int* herr, cudaStream_t st);
}  // namespace laph
