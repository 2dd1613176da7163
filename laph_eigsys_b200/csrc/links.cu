// links.cu -- boundary link layouts and plaquette reductions.
#include <cmath>

#include "links.cuh"
#include "su3.cuh"

namespace laph {

int links_to_soa(const double* in, int layout, int V3, double2* soa) {
  for (int s = 0; s < V3; ++s)
    for (int d = 0; d < 3; ++d)
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          const double* p;
          if (layout == LAPH_LAYOUT_ROWMAJOR) p = in + (((size_t)s * 3 + d) * 9 + 3 * a + b) * 2;
          else if (layout == LAPH_LAYOUT_EIGEN) p = in + (((size_t)s * 3 + d) * 9 + 3 * b + a) * 2;
          else if (layout == LAPH_LAYOUT_CONF) p = in + (size_t)s * 72 + (d + 1) * 18 + 6 * a + 2 * b;
          else {
            set_error("unknown link layout %d", layout);
            return LAPH_EINVAL;
          }
          soa[(size_t)(d * 9 + 3 * a + b) * V3 + s] = make_double2(p[0], p[1]);
        }
  return LAPH_OK;
}

int check_links_finite(const double* in, int layout, int V3, const char* who) {
  if (layout != LAPH_LAYOUT_ROWMAJOR && layout != LAPH_LAYOUT_EIGEN && layout != LAPH_LAYOUT_CONF) {
    set_error("%s: unknown link layout %d", who, layout);
    return LAPH_EINVAL;
  }
  // per site: 54 contiguous doubles (ROWMAJOR, EIGEN), or slots 1..3 of 72 (CONF)
  const size_t stride = layout == LAPH_LAYOUT_CONF ? 72 : 54, first = layout == LAPH_LAYOUT_CONF ? 18 : 0;
  long long bad = V3;
#pragma omp parallel for reduction(min : bad) schedule(static)
  for (long long s = 0; s < V3; ++s) {
    const double* p = in + (size_t)s * stride + first;
    bool ok = true;
    for (int e = 0; e < 54; ++e) ok &= std::isfinite(p[e]);
    if (!ok && s < bad) bad = s;
  }
  if (bad < V3) {
    set_error("%s: non-finite link value at site %lld", who, bad);
    return LAPH_EINVAL;
  }
  return LAPH_OK;
}

int soa_to_links(const double2* soa, int V3, int layout, double* out) {
  if (layout == LAPH_LAYOUT_CONF) {
    // the temporal slot is not held on the device: write the identity there
    for (int s = 0; s < V3; ++s)
      for (int k = 0; k < 18; ++k) out[(size_t)s * 72 + k] = (k == 0 || k == 8 || k == 16) ? 1.0 : 0.0;
  }
  for (int s = 0; s < V3; ++s)
    for (int d = 0; d < 3; ++d)
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          double* p;
          if (layout == LAPH_LAYOUT_ROWMAJOR) p = out + (((size_t)s * 3 + d) * 9 + 3 * a + b) * 2;
          else if (layout == LAPH_LAYOUT_EIGEN) p = out + (((size_t)s * 3 + d) * 9 + 3 * b + a) * 2;
          else if (layout == LAPH_LAYOUT_CONF) p = out + (size_t)s * 72 + (d + 1) * 18 + 6 * a + 2 * b;
          else {
            set_error("unknown link layout %d", layout);
            return LAPH_EINVAL;
          }
          const double2 v = soa[(size_t)(d * 9 + 3 * a + b) * V3 + s];
          p[0] = v.x;
          p[1] = v.y;
        }
  return LAPH_OK;
}

__global__ void k_links_to_soa(const double2* __restrict__ in, int layout, int V3, double2* __restrict__ soa) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 27LL * V3) return;
  const int e = (int)(t / V3), s = (int)(t - (long long)e * V3);  // e = dir*9 + 3a + b
  const int d = e / 9, ab = e - d * 9;
  const size_t src = layout == LAPH_LAYOUT_CONF ? (size_t)s * 36 + (d + 1) * 9 + ab : ((size_t)s * 3 + d) * 9 + ab;
  soa[t] = in[src];
}

int links_to_soa_device(const double* links, int layout, int V3, double2* soa, cudaStream_t st) {
  if (layout != LAPH_LAYOUT_ROWMAJOR && layout != LAPH_LAYOUT_CONF) {
    set_error("links_to_soa_device: layout %d not supported for device links", layout);
    return LAPH_EINVAL;
  }
  k_links_to_soa<<<ceil_div(27LL * V3, 256), 256, 0, st>>>(reinterpret_cast<const double2*>(links), layout, V3, soa);
  LAPH_CUDA_TRY(cudaGetLastError());
  LAPH_CUDA_TRY(cudaStreamSynchronize(st));
  return LAPH_OK;
}

// One CTA per timeslice, fixed reduction order (deterministic).
__global__ void __launch_bounds__(512) k_plaq_moments(const double2* __restrict__ Ub, Lat g, size_t ts_stride,
                                                      double* __restrict__ out) {
  const double2* U = Ub + blockIdx.x * ts_stride;
  double acc[4] = {0, 0, 0, 0};
  for (int s = threadIdx.x; s < g.V3; s += blockDim.x) {
    int x, y, z;
    site_xyz(g, s, x, y, z);
#pragma unroll 1
    for (int pl = 0; pl < 3; ++pl) {
      const int d1 = pl == 2 ? 1 : 0, d2 = pl == 0 ? 1 : 2;
      const int j = nb_up(g, x, y, z, d1);
      const int l = nb_up(g, x, y, z, d2);
      // P = U_d1(s) U_d2(s+d1) U_d1(s+d2)^dag U_d2(s)^dag
      const M3 a = m3_mul(ld_link(U, g.V3, s, d1), ld_link(U, g.V3, j, d2));
      const M3 b = m3_mul(ld_link(U, g.V3, s, d2), ld_link(U, g.V3, l, d1));
      // Re tr(a b^dag)
      double tr = 0.0;
#pragma unroll
      for (int e = 0; e < 9; ++e) tr += a.e[e].x * b.e[e].x + a.e[e].y * b.e[e].y;
      const double p = tr / 3.0;
      acc[0] += p;
      acc[1] += p * p;
      acc[2] += p * p * p;
      acc[3] += p * p * p * p;
    }
  }
  __shared__ double red[4][512];
#pragma unroll
  for (int k = 0; k < 4; ++k) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
#pragma unroll
      for (int k = 0; k < 4; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 4) out[blockIdx.x * 4 + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void k_plaq_finish(const double* __restrict__ mom, int nts, double inv_n, double* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nts) out[t] = mom[4 * t] * inv_n;
}

int plaquette_moments_batch(const double2* U, int L, int nts, double* out, cudaStream_t st) {
  const Lat g = make_lat(L);
  k_plaq_moments<<<nts, 512, 0, st>>>(U, g, (size_t)27 * g.V3, out);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}

int plaquette_batch(const double2* U, int L, int nts, double* out, cudaStream_t st) {
  const Lat g = make_lat(L);
  double* mom = nullptr;
  LAPH_CUDA_TRY(cudaMallocAsync(&mom, sizeof(double) * 4 * nts, st));
  k_plaq_moments<<<nts, 512, 0, st>>>(U, g, (size_t)27 * g.V3, mom);
  k_plaq_finish<<<ceil_div(nts, 128), 128, 0, st>>>(mom, nts, 1.0 / (3.0 * g.V3), out);
  LAPH_CUDA_TRY(cudaGetLastError());
  LAPH_CUDA_TRY(cudaFreeAsync(mom, st));
  return LAPH_OK;
}

}  // namespace laph
