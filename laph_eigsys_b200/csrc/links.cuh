// links.cuh -- link layout conversion at the boundary and per-timeslice
// plaquette reductions (links.cu).
#pragma once
#include "common.cuh"

namespace laph {
// Host: boundary layouts (LAPH_LAYOUT_*) <-> device site-minor order
// soa[(dir*9 + 3a + b)*V3 + site] (complex128).
int links_to_soa(const double* links, int layout, int V3, double2* soa);
int soa_to_links(const double2* soa, int V3, int layout, double* links);
// Host: LAPH_EINVAL (naming `who` and the first bad site) unless every spatial
// link entry of the host links in `layout` is finite; the temporal slot of
// LAPH_LAYOUT_CONF is not read.  NaN or Inf links would only turn into a solve
// that never converges, so they are refused before any device work.
int check_links_finite(const double* links, int layout, int V3, const char* who);
// Device: same reorder for links already in device memory (ROWMAJOR or CONF).
int links_to_soa_device(const double* links, int layout, int V3, double2* soa, cudaStream_t st);
// Device: average spatial plaquette of nts timeslices -> out[nts]
// (plaque_timeslice, modules/config_utils.cpp:388-426).
int plaquette_batch(const double2* U, int L, int nts, double* out, cudaStream_t st);
// Device: power sums of the per-(site, plane) plaquette p = Re tr P / 3:
// out[ts*4 + k] = sum p^(k+1) over 3*V3 values, k = 0..3.
int plaquette_moments_batch(const double2* U, int L, int nts, double* out, cudaStream_t st);
}  // namespace laph
