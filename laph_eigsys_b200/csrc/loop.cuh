// loop.cuh -- the solver's outer iteration on the device (loop.cu): the
// per-pass decisions the host loop makes between graph launches (filter
// degree, the learned window's check, convergence), made by small kernels
// inside one CUDA graph whose WHILE node repeats the pass while any problem
// is active, with IF nodes selecting the filter steps of the pass's degree.
#pragma once
#include "batch.cuh"

namespace laph {

// Device-side state of the outer loop (one per solver).
struct LoopState {
  int it;                        // outer iterations begun (the host loop's `it`)
  int m;                         // filter degree of the current pass
  int npass;                     // passes run
  int deg0;                      // learned first-pass degree cap (0: none)
  int direct;                    // every active problem runs the current pass directly (no S past step 2)
  double sv_steps;               // unlocked site-vector-steps filtered
  double fbytes[2];              // filter bytes (correction form, 72 B unit)
  double filt_ns;                // filter time from the global timer
  unsigned long long t_pass;     // global timer at the start of the current pass
  unsigned long long t_start;    // global timer at the start of the solve
  unsigned long long t_loop;     // ... when the loop begins (setup done)
  unsigned long long t_end;      // ... after the last pass
};

struct LoopParams {
  int mdeg;          // degree cap of every pass
  int max_it;        // passes run while it < max_it
  int kb;            // filter columns per CTA
  int mlp;           // window = learned: check its first pass
  double lbytes;     // filter link bytes per site per column block
  double lam_top;    // exact upper bound of the spectrum (12 or opts.lam_max)
  double cap_resid;  // degree cap while the largest wanted residual exceeds this
  double win_check;  // the learned window's check after its first pass
  double direct_resid;  // a problem's pass is direct while its largest wanted residual exceeds this (< 0: never)
};

// Stamp the global timer into *t.
int loop_stamp(unsigned long long* t, cudaStream_t st);
// Reset the counters; deg0 = max over problems of the learned degrees (wdeg may be null).
int loop_init(LoopState* ls, const int* wdeg, int np, cudaStream_t st);
// Begin a pass: it += 1, the learned window's check (it == 2), the degree m,
// each problem's direct flag, the counters, and the SWITCH handles of the
// filter steps n = 1..mdeg-1: 0 = a middle step (n < m - 1), 1 = the last step
// (n = m - 1), 2 / 3 = the same without S (n >= 3 of a pass every active
// problem runs directly), 4 = no step.
int loop_pass_begin(const ProbDesc* pd, ProbState* ps, int np, LoopState* ls, int* degs, double* lam_max0,
                    int* fallback, const cudaGraphConditionalHandle* steps, const LoopParams& lp, cudaStream_t st);
// End of the filter part of a pass: accumulate its time.
int loop_pass_end(LoopState* ls, cudaStream_t st);
// Loop condition for the next pass: any problem active and it + 1 < max_it.
int loop_cond(const LoopState* ls, const int* n_active, int max_it, cudaGraphConditionalHandle h, cudaStream_t st);
// Stamp the end of the loop (LoopState::t_end).
int loop_end(LoopState* ls, cudaStream_t st);
// *p = 0 (a kernel, so that it can sit in a conditional body).
int zero_int(int* p, cudaStream_t st);

}  // namespace laph
