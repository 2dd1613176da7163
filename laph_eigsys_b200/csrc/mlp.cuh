// mlp.cuh -- learned Chebyshev window: MLP sizes and device entry points (mlp.cu).
#pragma once
#include "batch.cuh"

namespace laph {
constexpr int kMlpIn = 16, kMlpH = 64, kMlpOut = 3;
constexpr int kMlpParams = kMlpH * kMlpIn + kMlpH + kMlpH * kMlpH + kMlpH + kMlpOut * kMlpH + kMlpOut;  // 5443
constexpr int kMlpNorm = 2 * kMlpIn + 2 * kMlpOut;  // feature mean/std, target mean/std
constexpr int kLanczosSteps = 10;
int mlp_forward(const float* P, const float* X, int n, float* H1, float* H2, float* O, cudaStream_t st);
// feats[np][16], bound[np] from the smeared links; scratch = the W block pool.
int features(const ProbDesc* pd, int np, const double2* U64, const double* plaq, double2* scratch, float* feats,
             double* bound, cudaStream_t st);
// model = params (kMlpParams) followed by the normalisation (kMlpNorm);
// work >= np * (kMlpIn + kMlpOut) floats; margin scales the predicted cut.
int window_infer(const ProbDesc* pd, ProbState* ps, int np, const float* feats, const float* model, float* work,
                 const double* bound, int* out_deg, double margin, cudaStream_t st);
// First-pass cut of the learned window = this x the predicted converged cut,
// unless laph_solve_opts.window_margin says otherwise.
constexpr double kWindowMargin = 1.4;
}  // namespace laph
