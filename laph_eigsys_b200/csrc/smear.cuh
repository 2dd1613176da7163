// smear.cuh -- FP64 device smearing entry points (see smear.cu).
#pragma once
#include "common.cuh"

namespace laph {
// U, Utmp: nts timeslices of links in site-minor order [ts][dir][9][V3]
// (complex128); dec: HYP scratch [ts][6][9][V3] (may be null for stout/APE).
// On return U holds the smeared links.
int smear_batch(double2* U, double2* Utmp, double2* dec, int L, int nts, int kind, double p1, double p2, int iters,
                int compat, cudaStream_t st);
}  // namespace laph
