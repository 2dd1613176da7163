// loop.cu -- kernels of the device-side outer loop (see loop.cuh).  They
// restate on the device the host loop of laph_solver_run: the degree of a
// pass (the cap that keeps the filter's amplification at lambda = 0 below
// 1e6 while the largest wanted residual exceeds cap_resid), the learned
// window's check after its first pass, the algorithmic-byte counters, and
// the convergence condition, so that one graph launch runs a whole solve.
#include <cmath>

#include "common.cuh"
#include "loop.cuh"

namespace laph {

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__global__ void k_loop_stamp(unsigned long long* t) { *t = gtimer(); }

__global__ void k_loop_init(LoopState* ls, const int* __restrict__ wdeg, int np) {
  __shared__ int s_max;
  if (threadIdx.x == 0) s_max = 0;
  __syncthreads();
  if (wdeg)
    for (int p = threadIdx.x; p < np; p += blockDim.x) atomicMax(&s_max, wdeg[p]);
  __syncthreads();
  if (threadIdx.x == 0) {
    ls->it = 0;
    ls->m = 0;
    ls->npass = 0;
    ls->deg0 = s_max;
    ls->direct = 0;
    ls->sv_steps = 0.0;
    ls->fbytes[0] = ls->fbytes[1] = 0.0;
    ls->filt_ns = 0.0;
    ls->t_loop = gtimer();
    ls->t_end = ls->t_loop;
  }
}

__global__ void k_loop_pass_begin(const ProbDesc* __restrict__ pd, ProbState* __restrict__ ps, int np, LoopState* ls,
                                  int* __restrict__ degs, double* __restrict__ lam_max0, int* __restrict__ fallback,
                                  const cudaGraphConditionalHandle* __restrict__ steps, LoopParams lp) {
  __shared__ int s_it, s_m, s_nact, s_ndir;
  __shared__ double s_sv, s_b0, s_b1;
  const int tid = threadIdx.x;
  if (tid == 0) {
    s_it = ls->it + 1;
    s_m = lp.mdeg;
    if (s_it == 1 && ls->deg0 > 0) s_m = min(s_m, max(2, ls->deg0));
    s_sv = s_b0 = s_b1 = 0.0;
    s_nact = s_ndir = 0;
  }
  __syncthreads();
  const int it = s_it;
  for (int p = tid; p < np; p += blockDim.x) {
    ProbState& S = ps[p];
    if (it == 1) lam_max0[p] = S.lam_max;
    // the learned window's check after its first pass (the host loop's rule)
    if (it == 2 && lp.mlp && S.active &&
        !(S.max_resid < lp.win_check && !S.chol_fail && isfinite(S.lam_cut))) {
      fallback[p] = 1;
      if (S.lam_max < lp.lam_top || !isfinite(S.lam_cut)) {
        double cut = isfinite(S.lam_cut) ? S.lam_cut : 0.5 * lp.lam_top;
        cut = fmin(fmax(cut, 1e-6), lp.lam_top - 1e-3);
        S.lam_max = lp.lam_top;
        S.lam_cut = cut;
        S.c_hop = 2.0 / (lp.lam_top - cut);
        S.c_diag = (lp.lam_top + cut - 12.0) / (lp.lam_top - cut);
      }
    }
    // a direct pass while the Ritz vectors are far from converged (FP32 rounding of T(B)V is harmless there),
    // until one fails to halve the residual
    if (S.active) {
      if (S.direct && !(S.max_resid < 0.5 * S.resid_begin)) S.direct_off = 1;
      S.resid_begin = S.max_resid;
    }
    S.direct = S.active && !S.direct_off && lp.direct_resid >= 0.0 && !(S.max_resid <= lp.direct_resid) ? 1 : 0;
    if (S.active) {
      atomicAdd(&s_nact, 1);
      if (S.direct) atomicAdd(&s_ndir, 1);
    }
    // degree cap while the Ritz vectors are still poor: amplification <= 1e6 at lambda = 0
    if (S.active && S.max_resid > lp.cap_resid) {
      const double tb0 = 1.0 + 2.0 * S.lam_cut / (S.lam_max - S.lam_cut);
      const double ratio = acosh(1e6) / acosh(fmax(tb0, 1.0 + 1e-12));
      const int m_safe = isfinite(ratio) ? (int)fmin(floor(ratio), 1e6) : 2;
      atomicMin(&s_m, max(2, m_safe));
    }
  }
  __syncthreads();
  const int m = s_m;
  const bool nos = s_nact > 0 && s_ndir == s_nact;
  // counters of this pass (the solver's filter byte model, per problem)
  for (int p = tid; p < np; p += blockDim.x) {
    const ProbState& S = ps[p];
    if (!S.active) continue;
    const ProbDesc d = pd[p];
    const int nl = S.nlock, nact = d.k - nl;
    const int nblk = (d.k + lp.kb - 1) / lp.kb - nl / lp.kb;
    double per = S.direct ? 72.0 : 0.0;  // a direct pass starts with S = FP32(V)
    for (int n = 1; n < m; ++n) {
      const int reads = n == 1 ? 1 : (n == 2 ? 2 : (nos ? 2 : 3));
      per += reads * 24.0 + (n == m - 1 ? 96.0 : 24.0);
    }
    atomicAdd(&s_sv, (double)d.V3 * nact * (m - 1));
    atomicAdd(&s_b0, (double)d.V3 * (nact * per + nl * 96.0 + (double)nblk * (m - 1) * lp.lbytes));
    atomicAdd(&s_b1, (double)d.V3 * (m - 1) * (nact * 72.0 + (double)nblk * lp.lbytes));
  }
  // the filter steps of this pass: n = 1..m-2 middle (0), n = m-1 the last (1), the same without S (2, 3) for
  // n >= 3 of an all-direct pass, none beyond (4: past the last branch of every SWITCH)
  for (int n = 1 + tid; n < lp.mdeg; n += blockDim.x) {
    const unsigned base = n < m - 1 ? 0u : (n == m - 1 ? 1u : 4u);
    cudaGraphSetConditional(steps[n], base < 2u && nos && n >= 3 ? base + 2u : base);
  }
  __syncthreads();
  if (tid == 0) {
    ls->it = it;
    ls->m = m;
    ls->direct = nos ? 1 : 0;
    degs[ls->npass] = m;
    ls->npass += 1;
    ls->sv_steps += s_sv;
    ls->fbytes[0] += s_b0;
    ls->fbytes[1] += s_b1;
    ls->t_pass = gtimer();
  }
}

__global__ void k_loop_pass_end(LoopState* ls) {
  const unsigned long long t = gtimer();
  ls->filt_ns += (double)(t - ls->t_pass);
}

__global__ void k_loop_cond(const LoopState* ls, const int* n_active, int max_it, cudaGraphConditionalHandle h) {
  const bool more = *n_active > 0 && ls->it + 1 < max_it;
  cudaGraphSetConditional(h, more ? 1u : 0u);
}

__global__ void k_loop_end(LoopState* ls) { ls->t_end = gtimer(); }

__global__ void k_zero_int(int* p) { *p = 0; }

int loop_stamp(unsigned long long* t, cudaStream_t st) {
  k_loop_stamp<<<1, 1, 0, st>>>(t);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}

int loop_init(LoopState* ls, const int* wdeg, int np, cudaStream_t st) {
  k_loop_init<<<1, 256, 0, st>>>(ls, wdeg, np);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}

int loop_pass_begin(const ProbDesc* pd, ProbState* ps, int np, LoopState* ls, int* degs, double* lam_max0,
                    int* fallback, const cudaGraphConditionalHandle* steps, const LoopParams& lp, cudaStream_t st) {
  k_loop_pass_begin<<<1, 256, 0, st>>>(pd, ps, np, ls, degs, lam_max0, fallback, steps, lp);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}

int loop_pass_end(LoopState* ls, cudaStream_t st) {
  k_loop_pass_end<<<1, 1, 0, st>>>(ls);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}

int loop_cond(const LoopState* ls, const int* n_active, int max_it, cudaGraphConditionalHandle h, cudaStream_t st) {
  k_loop_cond<<<1, 1, 0, st>>>(ls, n_active, max_it, h);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}

int loop_end(LoopState* ls, cudaStream_t st) {
  k_loop_end<<<1, 1, 0, st>>>(ls);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}

int zero_int(int* p, cudaStream_t st) {
  k_zero_int<<<1, 1, 0, st>>>(p);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}

}  // namespace laph
