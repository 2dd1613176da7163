// mlp.cu -- the learned Chebyshev window: a 16 -> 64 -> 64 -> 3 tanh MLP in
// FP32 with hand-written forward, backward and Adam kernels (training and
// inference on the device), plus the per-timeslice feature kernel.
//
// Parameter vector layout (kMlpParams floats):
//   W1[64][16] b1[64] W2[64][64] b2[64] W3[3][64] b3[3]
// A window model additionally carries the input standardisation (mean, std
// of the 16 features) and the output de-standardisation (mean, std of the 3
// targets); see laph_gpu.h.
#include <cmath>
#include <cstring>
#include <vector>

#include "batch.cuh"
#include "common.cuh"
#include "mlp.cuh"

namespace laph {

__host__ __device__ constexpr int o_W1() { return 0; }
__host__ __device__ constexpr int o_b1() { return kMlpH * kMlpIn; }
__host__ __device__ constexpr int o_W2() { return o_b1() + kMlpH; }
__host__ __device__ constexpr int o_b2() { return o_W2() + kMlpH * kMlpH; }
__host__ __device__ constexpr int o_W3() { return o_b2() + kMlpH; }
__host__ __device__ constexpr int o_b3() { return o_W3() + kMlpOut * kMlpH; }
static_assert(o_b3() + kMlpOut == kMlpParams, "parameter layout");

// Forward for n samples: one CTA of 64 threads per sample group, thread j
// owns hidden unit j.  Activations H1, H2 [n][64] and outputs O [n][3].
__global__ void __launch_bounds__(64) k_mlp_forward(const float* __restrict__ P, const float* __restrict__ X, int n,
                                                    float* __restrict__ H1, float* __restrict__ H2,
                                                    float* __restrict__ O) {
  __shared__ float sx[kMlpIn], sh1[kMlpH], sh2[kMlpH];
  const int j = threadIdx.x;
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    if (j < kMlpIn) sx[j] = X[(size_t)i * kMlpIn + j];
    __syncthreads();
    float z = P[o_b1() + j];
#pragma unroll
    for (int q = 0; q < kMlpIn; ++q) z = fmaf(P[o_W1() + j * kMlpIn + q], sx[q], z);
    const float h1 = tanhf(z);
    sh1[j] = h1;
    if (H1) H1[(size_t)i * kMlpH + j] = h1;
    __syncthreads();
    z = P[o_b2() + j];
    for (int q = 0; q < kMlpH; ++q) z = fmaf(P[o_W2() + j * kMlpH + q], sh1[q], z);
    const float h2 = tanhf(z);
    sh2[j] = h2;
    if (H2) H2[(size_t)i * kMlpH + j] = h2;
    __syncthreads();
    if (j < kMlpOut) {
      float o = P[o_b3() + j];
      for (int q = 0; q < kMlpH; ++q) o = fmaf(P[o_W3() + j * kMlpH + q], sh2[q], o);
      O[(size_t)i * kMlpOut + j] = o;
    }
    __syncthreads();
  }
}

// Backward of the mean-squared loss L = mean_{i,k} (O_ik - Y_ik)^2.  CTA g
// handles samples g, g + gridDim.x, ...; its gradient is accumulated in
// shared memory and written to partial row g (reduced in fixed order by
// k_mlp_reduce), so the gradient is deterministic.
__global__ void __launch_bounds__(64) k_mlp_backward(const float* __restrict__ P, const float* __restrict__ X,
                                                     const float* __restrict__ Y, int n, const float* __restrict__ H1,
                                                     const float* __restrict__ H2, const float* __restrict__ O,
                                                     float* __restrict__ gpart, float* __restrict__ lpart) {
  __shared__ float g[kMlpParams];
  __shared__ float sx[kMlpIn], sh1[kMlpH], sh2[kMlpH], sdo[kMlpOut], sd2[kMlpH];
  const int j = threadIdx.x;
  for (int e = j; e < kMlpParams; e += blockDim.x) g[e] = 0.f;
  float loss = 0.f;
  const float scale = 2.f / (float)(n * kMlpOut);
  __syncthreads();
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    if (j < kMlpIn) sx[j] = X[(size_t)i * kMlpIn + j];
    sh1[j] = H1[(size_t)i * kMlpH + j];
    sh2[j] = H2[(size_t)i * kMlpH + j];
    if (j < kMlpOut) {
      const float d = O[(size_t)i * kMlpOut + j] - Y[(size_t)i * kMlpOut + j];
      sdo[j] = scale * d;
      loss += d * d;
    }
    __syncthreads();
    // layer 3: dW3[k][j] += do_k h2_j ; db3 ; dh2_j = sum_k W3[k][j] do_k
    float dh2 = 0.f;
#pragma unroll
    for (int k = 0; k < kMlpOut; ++k) {
      g[o_W3() + k * kMlpH + j] += sdo[k] * sh2[j];
      dh2 = fmaf(P[o_W3() + k * kMlpH + j], sdo[k], dh2);
    }
    if (j < kMlpOut) g[o_b3() + j] += sdo[j];
    const float d2 = dh2 * (1.f - sh2[j] * sh2[j]);
    sd2[j] = d2;
    __syncthreads();
    // layer 2: dW2[j][q] += d2_j h1_q ; dh1_j = sum_r W2[r][j] d2_r
    for (int q = 0; q < kMlpH; ++q) g[o_W2() + j * kMlpH + q] += d2 * sh1[q];
    g[o_b2() + j] += d2;
    float dh1 = 0.f;
    for (int r = 0; r < kMlpH; ++r) dh1 = fmaf(P[o_W2() + r * kMlpH + j], sd2[r], dh1);
    const float d1 = dh1 * (1.f - sh1[j] * sh1[j]);
    // layer 1
#pragma unroll
    for (int q = 0; q < kMlpIn; ++q) g[o_W1() + j * kMlpIn + q] += d1 * sx[q];
    g[o_b1() + j] += d1;
    __syncthreads();
  }
  for (int e = j; e < kMlpParams; e += blockDim.x) gpart[(size_t)blockIdx.x * kMlpParams + e] = g[e];
  // loss: warp + block reduction
  for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
  __shared__ float sl[2];
  if ((j & 31) == 0) sl[j >> 5] = loss;
  __syncthreads();
  if (j == 0) lpart[blockIdx.x] = sl[0] + sl[1];
}

// Fixed-order reduction of the partial gradients, optional Adam step.
__global__ void k_mlp_reduce_adam(float* __restrict__ P, const float* __restrict__ gpart, int nblk,
                                  const float* __restrict__ lpart, float* __restrict__ grad, float* __restrict__ loss,
                                  float* __restrict__ m1, float* __restrict__ m2, float lr, float b1, float b2,
                                  float eps, int t, float inv_n_out, int do_adam) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e == 0 && loss) {
    float s = 0.f;
    for (int b = 0; b < nblk; ++b) s += lpart[b];
    *loss = s * inv_n_out;
  }
  if (e >= kMlpParams) return;
  float gsum = 0.f;
  for (int b = 0; b < nblk; ++b) gsum += gpart[(size_t)b * kMlpParams + e];
  if (grad) grad[e] = gsum;
  if (!do_adam) return;
  const float mm = b1 * m1[e] + (1.f - b1) * gsum;
  const float vv = b2 * m2[e] + (1.f - b2) * gsum * gsum;
  m1[e] = mm;
  m2[e] = vv;
  const float mh = mm / (1.f - powf(b1, (float)t));
  const float vh = vv / (1.f - powf(b2, (float)t));
  P[e] -= lr * mh / (sqrtf(vh) + eps);
}

// ---------------------------------------------------------------- features --
// One CTA (1024 threads) per problem: plaquette power sums of the smeared
// links and a 10-step FP64 Lanczos on -Delta from a fixed random start
// (vectors in the scratch block W), then the 10 Ritz values of the Lanczos
// tridiagonal (Jacobi on thread 0) and the upper bound theta_max + |beta s|.
// feats[p][16]: 0-3 plaquette mean / variance / skewness / excess kurtosis,
// 4-13 Ritz values / 12 ascending, 14 log(V3) / log(48^3), 15 k / dim.
// bound[p]: Lanczos upper bound of the spectrum.
__global__ void __launch_bounds__(1024) k_features(const ProbDesc* __restrict__ pd, const double2* __restrict__ U64,
                                                   const double* __restrict__ plaq, double2* __restrict__ scratch,
                                                   float* __restrict__ feats, double* __restrict__ bound) {
  const int p = blockIdx.x;
  const ProbDesc d = pd[p];
  const Lat g{d.L, d.L * d.L, d.V3};
  const double2* U = U64 + d.u64;
  double2* v0 = scratch + d.blk;  // three vectors of the problem's W block
  double2* v1 = v0 + d.dim;
  double2* w = v1 + d.dim;
  const int tid = threadIdx.x, nt = blockDim.x;
  __shared__ double red[32];
  __shared__ double s_alpha[kLanczosSteps], s_beta[kLanczosSteps];
  auto block_sum = [&](double x) {
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    __syncthreads();
    if ((tid & 31) == 0) red[tid >> 5] = x;
    __syncthreads();
    double s = 0.0;
    for (int q = 0; q < (nt >> 5); ++q) s += red[q];
    return s;
  };
  // start vector: counter hash, normalised
  double nrm = 0.0;
  for (int i = tid; i < d.dim; i += nt) {
    uint64_t z = (uint64_t)i * 0x9E3779B97F4A7C15ULL + 0x632BE59BD9B4E019ULL + (uint64_t)p * 0xD1B54A32D192ED03ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    const double a = ((z >> 11) * (1.0 / 9007199254740992.0)) - 0.5;
    const double b = (((z * 0x9E3779B97F4A7C15ULL) >> 11) * (1.0 / 9007199254740992.0)) - 0.5;
    v0[i] = make_double2(a, b);
    v1[i] = make_double2(0.0, 0.0);
    nrm += a * a + b * b;
  }
  nrm = block_sum(nrm);
  const double inv0 = 1.0 / sqrt(nrm);
  for (int i = tid; i < d.dim; i += nt) v0[i] = cscal(v0[i], inv0);
  __syncthreads();
  double2 *vc = v0, *vp = v1;
  double beta_prev = 0.0;
  for (int j = 0; j < kLanczosSteps; ++j) {
    // w = A vc - beta_prev vp ; alpha = <vc, w>
    double al = 0.0;
    for (int s = tid; s < d.V3; s += nt) {
      int sx, sy, sz;
      site_xyz(g, s, sx, sy, sz);
      double2 acc[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
      for (int mu = 0; mu < 3; ++mu) {
        const int u = nb_up(g, sx, sy, sz, mu), dn = nb_dn(g, sx, sy, sz, mu);
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) {
            cfma(acc[a], U[(size_t)(mu * 9 + 3 * a + b) * d.V3 + s], vc[3 * (size_t)u + b]);
            cfmac(acc[a], U[(size_t)(mu * 9 + 3 * b + a) * d.V3 + dn], vc[3 * (size_t)dn + b]);
          }
      }
      for (int a = 0; a < 3; ++a) {
        const double2 x = vc[3 * (size_t)s + a];
        const double2 y = vp[3 * (size_t)s + a];
        const double2 r = make_double2(6.0 * x.x - acc[a].x - beta_prev * y.x, 6.0 * x.y - acc[a].y - beta_prev * y.y);
        w[3 * (size_t)s + a] = r;
        al += x.x * r.x + x.y * r.y;
      }
    }
    al = block_sum(al);
    double bb = 0.0;
    for (int i = tid; i < d.dim; i += nt) {
      double2 r = w[i];
      const double2 x = vc[i];
      r.x -= al * x.x;
      r.y -= al * x.y;
      w[i] = r;
      bb += r.x * r.x + r.y * r.y;
    }
    bb = sqrt(block_sum(bb));
    if (tid == 0) {
      s_alpha[j] = al;
      s_beta[j] = bb;
    }
    const double ib = bb > 0.0 ? 1.0 / bb : 0.0;
    // next: vp <- w / beta (becomes the new current), old current becomes previous
    for (int i = tid; i < d.dim; i += nt) vp[i] = cscal(w[i], ib);
    __syncthreads();
    double2* t = vc;
    vc = vp;
    vp = t;
    beta_prev = bb;
  }
  if (tid == 0) {
    // Jacobi on the 10 x 10 tridiagonal
    constexpr int n = kLanczosSteps;
    double A[n][n], Q[n][n];
    for (int a = 0; a < n; ++a)
      for (int b = 0; b < n; ++b) {
        A[a][b] = (a == b) ? s_alpha[a] : ((b == a + 1) ? s_beta[a] : ((a == b + 1) ? s_beta[b] : 0.0));
        Q[a][b] = (a == b) ? 1.0 : 0.0;
      }
    for (int sweep = 0; sweep < 30; ++sweep) {
      double off = 0.0;
      for (int a = 0; a < n; ++a)
        for (int b = a + 1; b < n; ++b) off += A[a][b] * A[a][b];
      if (off < 1e-30) break;
      for (int a = 0; a < n - 1; ++a)
        for (int b = a + 1; b < n; ++b) {
          if (A[a][b] == 0.0) continue;
          const double tau = (A[b][b] - A[a][a]) / (2.0 * A[a][b]);
          const double tt = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
          const double c = 1.0 / sqrt(1.0 + tt * tt), s = tt * c;
          for (int k = 0; k < n; ++k) {
            const double ka = A[k][a], kb = A[k][b];
            A[k][a] = c * ka - s * kb;
            A[k][b] = s * ka + c * kb;
          }
          for (int k = 0; k < n; ++k) {
            const double ak = A[a][k], bk = A[b][k];
            A[a][k] = c * ak - s * bk;
            A[b][k] = s * ak + c * bk;
          }
          for (int k = 0; k < n; ++k) {
            const double qa = Q[k][a], qb = Q[k][b];
            Q[k][a] = c * qa - s * qb;
            Q[k][b] = s * qa + c * qb;
          }
        }
    }
    double th[n];
    int idx[n];
    for (int a = 0; a < n; ++a) {
      th[a] = A[a][a];
      idx[a] = a;
    }
    for (int a = 0; a < n; ++a)
      for (int b = a + 1; b < n; ++b)
        if (th[idx[b]] < th[idx[a]]) {
          const int t = idx[a];
          idx[a] = idx[b];
          idx[b] = t;
        }
    float* f = feats + (size_t)p * kMlpIn;
    const double* ps = plaq + 4 * (size_t)p;
    const double N = 3.0 * d.V3;
    const double mu = ps[0] / N;
    const double m2 = ps[1] / N - mu * mu;
    const double m3 = ps[2] / N - 3 * mu * ps[1] / N + 2 * mu * mu * mu;
    const double m4 = ps[3] / N - 4 * mu * ps[2] / N + 6 * mu * mu * ps[1] / N - 3 * mu * mu * mu * mu;
    const double sd = sqrt(fmax(m2, 1e-300));
    f[0] = (float)mu;
    f[1] = (float)m2;
    f[2] = (float)(m3 / (sd * sd * sd));
    f[3] = (float)(m4 / (m2 * m2) - 3.0);
    for (int a = 0; a < n; ++a) f[4 + a] = (float)(th[idx[a]] / 12.0);
    f[14] = (float)(log((double)d.V3) / log(48.0 * 48.0 * 48.0));
    f[15] = (float)((double)d.k / d.dim);
    const int top = idx[n - 1];
    bound[p] = th[top] + fabs(s_beta[n - 1] * Q[n - 1][top]);
  }
}

// Window inference: standardised features -> MLP -> (lam_cut, lam_max, deg)
// per problem, written into the problem state for the first filter pass.
//   lam_cut = margin x exp(prediction 0): target 0 is the log of the cut the
//             adaptive iteration converges to; the first pass starts above it
//             because its block is still a random one (margin calibrated on
//             training lattices, laph_solve_opts.window_margin);
//   lam_max stays the exact bound 12 of the spectrum of -Delta (or the fixed
//             one): prediction 1 learns the 10-step Lanczos estimate of the
//             top, which lies well below the true top (9.3-10.6 against
//             11.5+ on 16^3-32^3 smeared fields), and a window whose top is
//             below the spectrum's lets T_m amplify the highest eigenvectors
//             past the wanted ones -- solves with it did not converge in 300
//             passes -- so it is not used;
//   degree  = prediction 2, clamped to [8, 64], written to out_deg.
__global__ void k_window_apply(const ProbDesc* __restrict__ pd, ProbState* __restrict__ ps, int np,
                               const float* __restrict__ O, const float* __restrict__ norm,
                               const double* __restrict__ bound, int* __restrict__ out_deg, double margin) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const float* om = norm + 2 * kMlpIn;  // output mean[3], std[3]
  const double y0 = O[p * kMlpOut + 0] * om[3] + om[0];
  const double y2 = O[p * kMlpOut + 2] * om[5] + om[2];
  (void)bound;
  ProbState& S = ps[p];
  const double cut = exp(y0) * margin;
  S.lam_cut = isfinite(cut) ? fmin(fmax(cut, 1e-3), S.lam_max - 1e-3) : 0.5 * S.lam_max;
  out_deg[p] = isfinite(y2) ? (int)lrint(fmin(64.0, fmax(8.0, y2))) : 64;
}

// Standardise features with the model's mean/std.
__global__ void k_standardise(const float* __restrict__ f, const float* __restrict__ norm, int n,
                              float* __restrict__ x) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n * kMlpIn) return;
  const int q = e % kMlpIn;
  x[e] = (f[e] - norm[q]) / norm[kMlpIn + q];
}

// ------------------------------------------------------------- launchers --
int mlp_forward(const float* P, const float* X, int n, float* H1, float* H2, float* O, cudaStream_t st) {
  k_mlp_forward<<<std::min(n, 4096), 64, 0, st>>>(P, X, n, H1, H2, O);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}

int features(const ProbDesc* pd, int np, const double2* U64, const double* plaq, double2* scratch, float* feats,
             double* bound, cudaStream_t st) {
  k_features<<<np, 1024, 0, st>>>(pd, U64, plaq, scratch, feats, bound);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}

int window_infer(const ProbDesc* pd, ProbState* ps, int np, const float* feats, const float* model, float* work,
                 const double* bound, int* out_deg, double margin, cudaStream_t st) {
  // model = [params | norm(16 mean, 16 std, 3 mean, 3 std)]
  float* X = work;
  float* O = work + (size_t)np * kMlpIn;
  k_standardise<<<ceil_div((long long)np * kMlpIn, 256), 256, 0, st>>>(feats, model + kMlpParams, np, X);
  LAPH_TRY(mlp_forward(model, X, np, nullptr, nullptr, O, st));
  k_window_apply<<<ceil_div(np, 128), 128, 0, st>>>(pd, ps, np, O, model + kMlpParams, bound, out_deg, margin);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}

}  // namespace laph

using namespace laph;

namespace {
struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};
int dalloc_f(DevBuf& b, size_t n) {
  if (cudaMalloc(&b.p, n * sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    set_error("mlp: device allocation failed");
    return LAPH_ENOMEM;
  }
  return LAPH_OK;
}
}  // namespace

extern "C" {

int laph_mlp_nparams(void) { return kMlpParams; }

int laph_mlp_forward(const float* params, const float* X, int n, float* out, int device) {
  if (!params || !X || !out || n < 1) {
    set_error("laph_mlp_forward: bad argument");
    return LAPH_EINVAL;
  }
  LAPH_CUDA_TRY(cudaSetDevice(device));
  DevBuf P, dX, dO;
  LAPH_TRY(dalloc_f(P, kMlpParams));
  LAPH_TRY(dalloc_f(dX, (size_t)n * kMlpIn));
  LAPH_TRY(dalloc_f(dO, (size_t)n * kMlpOut));
  LAPH_CUDA_TRY(cudaMemcpy(P.p, params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice));
  LAPH_CUDA_TRY(cudaMemcpy(dX.p, X, sizeof(float) * n * kMlpIn, cudaMemcpyHostToDevice));
  LAPH_TRY(mlp_forward((float*)P.p, (float*)dX.p, n, nullptr, nullptr, (float*)dO.p, 0));
  LAPH_CUDA_TRY(cudaMemcpy(out, dO.p, sizeof(float) * n * kMlpOut, cudaMemcpyDeviceToHost));
  return LAPH_OK;
}

// Gradient of the mean-squared loss at params (for the gradient check), or
// `epochs` full-batch Adam steps from params (training; params updated).
static int mlp_run(float* params, const float* X, const float* Y, int n, int epochs, float lr, float* grad_out,
                   float* loss_out, int device) {
  if (!params || !X || !Y || n < 1) {
    set_error("laph_mlp: bad argument");
    return LAPH_EINVAL;
  }
  LAPH_CUDA_TRY(cudaSetDevice(device));
  const int nblk = std::min(n, 148);
  DevBuf P, dX, dY, H1, H2, O, gp, lp, g, l, m1, m2;
  LAPH_TRY(dalloc_f(P, kMlpParams));
  LAPH_TRY(dalloc_f(dX, (size_t)n * kMlpIn));
  LAPH_TRY(dalloc_f(dY, (size_t)n * kMlpOut));
  LAPH_TRY(dalloc_f(H1, (size_t)n * kMlpH));
  LAPH_TRY(dalloc_f(H2, (size_t)n * kMlpH));
  LAPH_TRY(dalloc_f(O, (size_t)n * kMlpOut));
  LAPH_TRY(dalloc_f(gp, (size_t)nblk * kMlpParams));
  LAPH_TRY(dalloc_f(lp, nblk));
  LAPH_TRY(dalloc_f(g, kMlpParams));
  LAPH_TRY(dalloc_f(l, 1));
  LAPH_TRY(dalloc_f(m1, kMlpParams));
  LAPH_TRY(dalloc_f(m2, kMlpParams));
  LAPH_CUDA_TRY(cudaMemcpy(P.p, params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice));
  LAPH_CUDA_TRY(cudaMemcpy(dX.p, X, sizeof(float) * n * kMlpIn, cudaMemcpyHostToDevice));
  LAPH_CUDA_TRY(cudaMemcpy(dY.p, Y, sizeof(float) * n * kMlpOut, cudaMemcpyHostToDevice));
  LAPH_CUDA_TRY(cudaMemset(m1.p, 0, sizeof(float) * kMlpParams));
  LAPH_CUDA_TRY(cudaMemset(m2.p, 0, sizeof(float) * kMlpParams));
  const int steps = epochs > 0 ? epochs : 1;
  for (int t = 1; t <= steps; ++t) {
    k_mlp_forward<<<std::min(n, 4096), 64>>>((float*)P.p, (float*)dX.p, n, (float*)H1.p, (float*)H2.p, (float*)O.p);
    k_mlp_backward<<<nblk, 64>>>((float*)P.p, (float*)dX.p, (float*)dY.p, n, (float*)H1.p, (float*)H2.p,
                                 (float*)O.p, (float*)gp.p, (float*)lp.p);
    k_mlp_reduce_adam<<<ceil_div(kMlpParams, 256), 256>>>((float*)P.p, (float*)gp.p, nblk, (float*)lp.p,
                                                          (float*)g.p, (float*)l.p, (float*)m1.p, (float*)m2.p, lr,
                                                          0.9f, 0.999f, 1e-8f, t, 1.f / (float)(n * kMlpOut),
                                                          epochs > 0);
    LAPH_CUDA_TRY(cudaGetLastError());
  }
  LAPH_CUDA_TRY(cudaDeviceSynchronize());
  if (grad_out) LAPH_CUDA_TRY(cudaMemcpy(grad_out, g.p, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost));
  if (loss_out) LAPH_CUDA_TRY(cudaMemcpy(loss_out, l.p, sizeof(float), cudaMemcpyDeviceToHost));
  if (epochs > 0) LAPH_CUDA_TRY(cudaMemcpy(params, P.p, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost));
  return LAPH_OK;
}

int laph_mlp_grad(const float* params, const float* X, const float* Y, int n, float* grad, float* loss, int device) {
  std::vector<float> p(params, params + kMlpParams);
  return mlp_run(p.data(), X, Y, n, 0, 0.f, grad, loss, device);
}

int laph_mlp_train(float* params, const float* X, const float* Y, int n, int epochs, float lr, float* loss, int device) {
  if (epochs < 1) {
    set_error("laph_mlp_train: epochs must be >= 1");
    return LAPH_EINVAL;
  }
  return mlp_run(params, X, Y, n, epochs, lr, nullptr, loss, device);
}

}  // extern "C"
