// smear.cu -- FP64 smearing of the spatial links of a timeslice on the device:
// stout, APE and 3D HYP, restating Tslice::smearing_stout / smearing_ape /
// smearing_hyp (modules/timeslice.cpp:145-369) with one thread per link.
//
// Every kernel reads the links of the previous iteration and writes a
// separate output (Jacobi-style, all links updated at once), exactly as the
// reference's eigen_timeslice_ts temporaries do.  A batch of nts timeslices
// of equal volume is processed by one launch (grid.y = timeslice).
#include "smear.cuh"
#include "su3.cuh"

namespace laph {

// Staple sum of smearing_stout / smearing_ape (timeslice.cpp:159-174).
// compat: reference backward staple U_nd(x-nd)^dag U_dir(x-nd) U_dir(x-nd+dir)
// (timeslice.cpp:171-172); otherwise the gauge-covariant U_nd(x-nd+dir).
__device__ __forceinline__ M3 staple_sum(const double2* __restrict__ U, const Lat& g, int x, int y, int z, int s,
                                         int dir, bool compat) {
  M3 st = m3_zero();
#pragma unroll 1
  for (int nd = 0; nd < 3; ++nd) {
    if (nd == dir) continue;
    const int s_up_nd = nb_up(g, x, y, z, nd);
    const int s_up_dir = nb_up(g, x, y, z, dir);
    // forward: U_nd(x) U_dir(x+nd) U_nd(x+dir)^dag
    M3 t = m3_mul(ld_link(U, g.V3, s_up_nd, dir), m3_adj(ld_link(U, g.V3, s_up_dir, nd)));
    m3_acc(st, m3_mul(ld_link(U, g.V3, s, nd), t));
    // backward
    const int s_dn = nb_dn(g, x, y, z, nd);
    const int s_dn_up = site_up(g, s_dn, dir);
    const M3 third = ld_link(U, g.V3, s_dn_up, compat ? dir : nd);
    t = m3_mul(ld_link(U, g.V3, s_dn, dir), third);
    m3_acc(st, m3_adj_mul(ld_link(U, g.V3, s_dn, nd), t));
  }
  return st;
}

__global__ void __launch_bounds__(128) k_stout(const double2* __restrict__ Uin, double2* __restrict__ Uout, Lat g,
                                               double rho, int compat, size_t ts_stride) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= 3 * g.V3) return;
  const int dir = tid / g.V3, s = tid - dir * g.V3;
  const double2* U = Uin + blockIdx.y * ts_stride;
  int x, y, z;
  site_xyz(g, s, x, y, z);
  const M3 st = staple_sum(U, g, x, y, z, s, dir, compat != 0);
  const M3 u = ld_link(U, g.V3, s, dir);
  // Omega = (rho/4) C U^dag (timeslice.cpp:175)
  M3 om = m3_mul_adj(st, u);
#pragma unroll
  for (int i = 0; i < 9; ++i) om.e[i] = cscal(om.e[i], rho / 4.0);
  // q = (Omega^dag - Omega)/2 - tr(Omega^dag - Omega)/6 (timeslice.cpp:176-177); exp(-q) = exp(iH), H = i q
  M3 d;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) d.e[3 * i + j] = csub(cconj(om.e[3 * j + i]), om.e[3 * i + j]);
  const double2 tr = cadd(cadd(d.e[0], d.e[4]), d.e[8]);
  M3 H;
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    double2 q = cscal(d.e[i], 0.5);
    if (i == 0 || i == 4 || i == 8) q = csub(q, cscal(tr, 1.0 / 6.0));
    H.e[i] = make_double2(-q.y, q.x);  // i*q
  }
  st_link(Uout + blockIdx.y * ts_stride, g.V3, s, dir, m3_mul(expiH(H), u));
}

__global__ void __launch_bounds__(128) k_ape(const double2* __restrict__ Uin, double2* __restrict__ Uout, Lat g,
                                             double alpha, int compat, size_t ts_stride) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= 3 * g.V3) return;
  const int dir = tid / g.V3, s = tid - dir * g.V3;
  const double2* U = Uin + blockIdx.y * ts_stride;
  int x, y, z;
  site_xyz(g, s, x, y, z);
  const M3 st = staple_sum(U, g, x, y, z, s, dir, compat != 0);
  // (1-alpha) U + alpha/4 C, then projection (timeslice.cpp:225, :230)
  const M3 m = m3_lin(ld_link(U, g.V3, s, dir), 1.0 - alpha, st, alpha / 4.0);
  st_link(Uout + blockIdx.y * ts_stride, g.V3, s, dir, proj_su3(m));
}

// HYP level 1 (timeslice.cpp:263-306): decorated link of direction dir with
// staples in the perpendicular direction p, stored at slot dir (p = first
// perpendicular) or dir+3 (second), matching decor() (timeslice.cpp:125-140).
__global__ void __launch_bounds__(128) k_hyp1(const double2* __restrict__ Uin, double2* __restrict__ dec, Lat g,
                                              double alpha2, size_t ts_stride, size_t dec_stride) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= 6 * g.V3) return;
  const int slot = tid / g.V3, s = tid - slot * g.V3;
  const int dir = slot % 3;
  const int which = slot / 3;
  // get_dirs (timeslice.cpp:106-122)
  const int p = (dir == 0) ? (which == 0 ? 1 : 2) : (dir == 1 ? (which == 0 ? 0 : 2) : (which == 0 ? 0 : 1));
  const double2* U = Uin + blockIdx.y * ts_stride;
  int x, y, z;
  site_xyz(g, s, x, y, z);
  const int s_up_p = nb_up(g, x, y, z, p);
  const int s_up_dir = nb_up(g, x, y, z, dir);
  M3 inner = m3_mul(ld_link(U, g.V3, s, p),
                    m3_mul(ld_link(U, g.V3, s_up_p, dir), m3_adj(ld_link(U, g.V3, s_up_dir, p))));
  const int s_dn = nb_dn(g, x, y, z, p);
  const int s_dn_up = site_up(g, s_dn, dir);
  m3_acc(inner, m3_adj_mul(ld_link(U, g.V3, s_dn, p), m3_mul(ld_link(U, g.V3, s_dn, dir), ld_link(U, g.V3, s_dn_up, p))));
  const M3 stac = m3_lin(ld_link(U, g.V3, s, dir), 1.0 - alpha2, inner, alpha2 / 2.0);
  const M3 r = proj_su3(stac);
  double2* D = dec + blockIdx.y * dec_stride;
#pragma unroll
  for (int e = 0; e < 9; ++e) D[(size_t)(slot * 9 + e) * g.V3 + s] = r.e[e];
}

__device__ __forceinline__ int hyp_decor(int dir, int plane) {
  if (dir == 0) return plane == 1 ? 0 : 3;
  if (dir == 1) return plane == 0 ? 1 : 4;
  return plane == 0 ? 2 : 5;
}

// HYP level 2 + projection (timeslice.cpp:311-357).
__global__ void __launch_bounds__(128) k_hyp2(const double2* __restrict__ Uin, const double2* __restrict__ dec,
                                              double2* __restrict__ Uout, Lat g, double alpha1, size_t ts_stride,
                                              size_t dec_stride) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= 3 * g.V3) return;
  const int dir = tid / g.V3, s = tid - dir * g.V3;
  const double2* U = Uin + blockIdx.y * ts_stride;
  const double2* D = dec + blockIdx.y * dec_stride;
  int x, y, z;
  site_xyz(g, s, x, y, z);
  M3 outer = m3_zero();
#pragma unroll 1
  for (int nd = 0; nd < 3; ++nd) {
    if (nd == dir) continue;
    const int plane = ((dir + 1) ^ (nd + 1)) - 1;
    const int a = hyp_decor(nd, plane), b = hyp_decor(dir, plane);
    const int s_up_nd = nb_up(g, x, y, z, nd);
    const int s_up_dir = nb_up(g, x, y, z, dir);
    m3_acc(outer, m3_mul(ld_link(D, g.V3, s, a), m3_mul(ld_link(D, g.V3, s_up_nd, b), m3_adj(ld_link(D, g.V3, s_up_dir, a)))));
    const int s_dn = nb_dn(g, x, y, z, nd);
    const int s_dn_up = site_up(g, s_dn, dir);
    m3_acc(outer, m3_adj_mul(ld_link(D, g.V3, s_dn, a), m3_mul(ld_link(D, g.V3, s_dn, b), ld_link(D, g.V3, s_dn_up, a))));
  }
  const M3 m = m3_lin(ld_link(U, g.V3, s, dir), 1.0 - alpha1, outer, alpha1 / 4.0);
  st_link(Uout + blockIdx.y * ts_stride, g.V3, s, dir, proj_su3(m));
}

// ld_link with slot index > 2 addresses the decorated-link array (6 slots).

int smear_batch(double2* U, double2* Utmp, double2* dec, int L, int nts, int kind, double p1, double p2, int iters,
                int compat, cudaStream_t st) {
  const Lat g = make_lat(L);
  const size_t ts_stride = (size_t)27 * g.V3;
  const size_t dec_stride = (size_t)54 * g.V3;
  if (kind == LAPH_SMEAR_NONE || iters <= 0) return LAPH_OK;
  const dim3 blk(128);
  for (int it = 0; it < iters; ++it) {
    if (kind == LAPH_SMEAR_STOUT) {
      k_stout<<<dim3(ceil_div(3LL * g.V3, 128), nts), blk, 0, st>>>(U, Utmp, g, p1, compat, ts_stride);
    } else if (kind == LAPH_SMEAR_APE) {
      k_ape<<<dim3(ceil_div(3LL * g.V3, 128), nts), blk, 0, st>>>(U, Utmp, g, p1, compat, ts_stride);
    } else if (kind == LAPH_SMEAR_HYP) {
      if (!dec) {
        set_error("smear_batch: HYP needs the decorated-link scratch");
        return LAPH_EINVAL;
      }
      k_hyp1<<<dim3(ceil_div(6LL * g.V3, 128), nts), blk, 0, st>>>(U, dec, g, p2, ts_stride, dec_stride);
      k_hyp2<<<dim3(ceil_div(3LL * g.V3, 128), nts), blk, 0, st>>>(U, dec, Utmp, g, p1, ts_stride, dec_stride);
    } else {
      set_error("smear_batch: unknown smearing kind %d", kind);
      return LAPH_EINVAL;
    }
    LAPH_CUDA_TRY(cudaGetLastError());
    LAPH_CUDA_TRY(cudaMemcpyAsync(U, Utmp, sizeof(double2) * ts_stride * nts, cudaMemcpyDeviceToDevice, st));
  }
  return LAPH_OK;
}

}  // namespace laph
