// stencil64.cu -- FP64 covariant-Laplacian stencils.
//
// One kernel covers the reference's tv2 (modules/shell_matop.cpp:16-103) and
// one step of tv_iter's Chebyshev recurrence (:136-168):
//     y = c_hop * hop(x) + c_diag * x + c_z * z,
//     hop(x)(s) = sum_mu U_mu(s) x(s+mu) + U_mu(s-mu)^dag x(s-mu),
// so  B x          : c_hop = c,  c_diag = a - 6c, c_z = 0
//     2 B x - z    : c_hop = 2c, c_diag = 2(a-6c), c_z = -1
//     (-Delta) x   : c_hop = -1, c_diag = 6.
// Vectors keep the reference layout (complex128, index 3*site + colour); a
// block of ncol vectors is column-major with column stride ld.  One thread per
// (site, column); consecutive threads take consecutive sites so every
// 48-byte site vector and every link element is read coalesced.
#include "stencil64.cuh"
#include "su3.cuh"

namespace laph {

template <bool HAS_Z>
__global__ void __launch_bounds__(128) k_hop64(const double2* __restrict__ U, Lat g, const double2* __restrict__ X,
                                               const double2* __restrict__ Z, double2* __restrict__ Y, size_t ld,
                                               double c_hop, double c_diag, double c_z) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V3) return;
  const size_t col = (size_t)blockIdx.y * ld;
  const double2* x = X + col;
  int sx, sy, sz;
  site_xyz(g, s, sx, sy, sz);
  double2 acc[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
#pragma unroll
  for (int mu = 0; mu < 3; ++mu) {
    const int up = nb_up(g, sx, sy, sz, mu);
    const int dn = nb_dn(g, sx, sy, sz, mu);
    double2 xu[3], xd[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      xu[b] = __ldg(x + 3 * (size_t)up + b);
      xd[b] = __ldg(x + 3 * (size_t)dn + b);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        cfma(acc[a], __ldg(U + (size_t)(mu * 9 + 3 * a + b) * g.V3 + s), xu[b]);
        cfmac(acc[a], __ldg(U + (size_t)(mu * 9 + 3 * b + a) * g.V3 + dn), xd[b]);
      }
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double2 xs = __ldg(x + 3 * (size_t)s + a);
    double2 r = make_double2(c_hop * acc[a].x + c_diag * xs.x, c_hop * acc[a].y + c_diag * xs.y);
    if (HAS_Z) {
      const double2 zz = __ldg(Z + col + 3 * (size_t)s + a);
      r.x += c_z * zz.x;
      r.y += c_z * zz.y;
    }
    Y[col + 3 * (size_t)s + a] = r;
  }
}

int hop64(const double2* U, int L, const double2* X, const double2* Z, double2* Y, size_t ld, int ncol, double c_hop,
          double c_diag, double c_z, cudaStream_t st) {
  const Lat g = make_lat(L);
  const dim3 grid(ceil_div(g.V3, 128), ncol);
  if (Z)
    k_hop64<true><<<grid, 128, 0, st>>>(U, g, X, Z, Y, ld, c_hop, c_diag, c_z);
  else
    k_hop64<false><<<grid, 128, 0, st>>>(U, g, X, nullptr, Y, ld, c_hop, c_diag, 0.0);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}

// y = T_deg(B) x, B = c(hop - 6) + a (tv_iter, shell_matop.cpp:136-168).
// tmp must hold 2 vectors of dim = 3*V3 (column stride ld).
int cheb64(const double2* U, int L, double lam_l, double lam_c, int deg, const double2* x, double2* y, double2* tmp,
           size_t ld, int ncol, cudaStream_t st) {
  const double c = 2.0 / (lam_l - lam_c);
  const double a = 1.0 + c * lam_c;
  if (deg <= 1) return hop64(U, L, x, nullptr, y, ld, ncol, c, a - 6.0 * c, 0.0, st);
  // T_n lives in bufs[idx(n)], idx(n) = (2 - (deg - n)) mod 3, so T_deg lands
  // in y and three consecutive T's never share a buffer.
  double2* bufs[3] = {tmp, tmp + ld * ncol, y};
  auto idx = [deg](int n) { return (((2 - (deg - n)) % 3) + 3) % 3; };
  LAPH_TRY(hop64(U, L, x, nullptr, bufs[idx(1)], ld, ncol, c, a - 6.0 * c, 0.0, st));
  for (int n = 2; n <= deg; ++n) {
    const double2* prev = (n == 2) ? x : bufs[idx(n - 2)];
    LAPH_TRY(hop64(U, L, bufs[idx(n - 1)], prev, bufs[idx(n)], ld, ncol, 2.0 * c, 2.0 * (a - 6.0 * c), -1.0, st));
  }
  return LAPH_OK;
}

}  // namespace laph
