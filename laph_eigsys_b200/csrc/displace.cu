// displace.cu -- the covariant displacement of eigenvector blocks, the next
// step of distillation operators after the eigensystem
// (right_displacement_one_dir, modules/config_utils.cpp:344-382):
//
//   W_i(x) = 1/2 ( U_dir(x) V_i(x + dir) - U_dir(x - dir)^dag V_i(x - dir) )
//
// for every column i of a column-major complex128 block [3 V3][nev] (index
// 3 site + colour).  k_displace: one thread per site walks kDispCols columns
// with the site's two FP64 links (forward U_dir(x), backward U_dir(x-dir)) in
// 72 registers, read once per column block; neighbour vector rows come from
// L1/L2.  HBM-bound: algorithmic bytes per site and column 48 (V) + 48 (W),
// plus 288 B of links per site per column block.
#include "batch.cuh"
#include "common.cuh"

struct laph_ctx;

namespace laph {
int ctx_device_links(laph_ctx* c, const double2** U, int* L, double* lam_l, double* lam_c, int* deg, cudaStream_t* st,
                     int* dev);

namespace {

constexpr int kDispCols = 16;

__global__ void __launch_bounds__(128) k_displace(const double2* __restrict__ U, int L, int dir, int nev, long long ldv,
                                                  const double2* __restrict__ V, double2* __restrict__ W, int cm) {
  const Lat g{L, L * L, L * L * L};
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V3) return;
  const int j0 = blockIdx.y * kDispCols, j1 = min(nev, j0 + kDispCols);
  int sx, sy, sz;
  site_xyz(g, s, sx, sy, sz);
  const int up = nb_up(g, sx, sy, sz, dir), dn = nb_dn(g, sx, sy, sz, dir);
  double2 uf[9], ub[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) {
    uf[e] = __ldg(U + (size_t)(dir * 9 + e) * g.V3 + s);
    ub[e] = __ldg(U + (size_t)(dir * 9 + e) * g.V3 + dn);
  }
  for (int j = j0; j < j1; ++j) {
    const double2* v = V + (size_t)j * ldv;
    double2 vu[3], vd[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      // input 3*site + colour, or colour-major (cm: colour*V3 + site, the solver's own blocks)
      vu[b] = __ldg(v + (cm ? (size_t)b * g.V3 + up : 3 * (size_t)up + b));
      vd[b] = __ldg(v + (cm ? (size_t)b * g.V3 + dn : 3 * (size_t)dn + b));
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double2 f = make_double2(0.0, 0.0), bk = make_double2(0.0, 0.0);
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        cfma(f, uf[3 * a + b], vu[b]);   // U(x)[a][b] V(x+dir)[b]
        cfmac(bk, ub[3 * b + a], vd[b]); // conj(U(x-dir)[b][a]) V(x-dir)[b]
      }
      W[(size_t)j * ldv + 3 * (size_t)s + a] = make_double2(0.5 * (f.x - bk.x), 0.5 * (f.y - bk.y));
    }
  }
}

}  // namespace

// W = displacement of V (device blocks, column stride ldv) along dir with site-minor FP64 links U.
// cm: V colour-major (colour*V3 + site); W is always 3*site + colour.
int displace_device(const double2* U, int L, int dir, int nev, long long ldv, const double2* V, double2* W, int cm,
                    cudaStream_t st) {
  const int V3 = L * L * L;
  const dim3 grid((V3 + 127) / 128, (nev + kDispCols - 1) / kDispCols);
  k_displace<<<grid, 128, 0, st>>>(U, L, dir, nev, ldv, V, W, cm);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}

}  // namespace laph

using namespace laph;

extern "C" int laph_displace(laph_ctx* ctx, int dir, const double* V, double* W, int nev, int on_device) {
  const double2* U = nullptr;
  int L = 0, deg = 0, dev = 0;
  double lam_l = 0, lam_c = 0;
  cudaStream_t st = nullptr;
  if (!V || !W || nev < 1 || dir < 0 || dir > 2) {
    set_error("laph_displace: bad argument (need V, W, nev >= 1 and dir in 0..2)");
    return LAPH_EINVAL;
  }
  LAPH_TRY(ctx_device_links(ctx, &U, &L, &lam_l, &lam_c, &deg, &st, &dev));
  const long long dim = 3LL * L * L * L;
  if (on_device) {
    if (V == W) {
      set_error("laph_displace: V and W must not overlap");
      return LAPH_EINVAL;
    }
    LAPH_TRY(displace_device(U, L, dir, nev, dim, reinterpret_cast<const double2*>(V), reinterpret_cast<double2*>(W),
                             0, st));
    LAPH_CUDA_TRY(cudaStreamSynchronize(st));
    return LAPH_OK;
  }
  double2 *dV = nullptr, *dW = nullptr;
  if (cudaMalloc(&dV, sizeof(double2) * dim * nev) != cudaSuccess ||
      cudaMalloc(&dW, sizeof(double2) * dim * nev) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(dV);
    set_error("laph_displace: device allocation failed");
    return LAPH_ENOMEM;
  }
  int rc = LAPH_OK;
  if (cudaMemcpyAsync(dV, V, sizeof(double2) * dim * nev, cudaMemcpyHostToDevice, st) != cudaSuccess) {
    rc = LAPH_ECUDA;
  } else {
    rc = displace_device(U, L, dir, nev, dim, dV, dW, 0, st);
    if (rc == LAPH_OK && cudaMemcpyAsync(W, dW, sizeof(double2) * dim * nev, cudaMemcpyDeviceToHost, st) != cudaSuccess)
      rc = LAPH_ECUDA;
  }
  if (cudaStreamSynchronize(st) != cudaSuccess && rc == LAPH_OK) rc = LAPH_ECUDA;
  if (rc == LAPH_ECUDA) set_error("laph_displace: %s", cudaGetErrorString(cudaGetLastError()));
  cudaFree(dV);
  cudaFree(dW);
  return rc;
}
