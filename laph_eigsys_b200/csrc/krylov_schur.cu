// krylov_schur.cu -- the "plain" form: SLEPc-style Krylov-Schur (EPS_HEP,
// EPS_LARGEST_MAGNITUDE) on T_DEG(B), driving the GPU MatShell product
// exactly as SLEPc's EPSSolve drives MatMult_Laplacian2D in the reference
// (src/ev_ts.cpp:231-263, modules/shell_matop.cpp:226-244).
//
// Algorithm (SLEPc 3.12 krylovschur, symmetric variant, restated): expand a
// Lanczos basis to ncv = max(2 nev, nev + 15) vectors with full classical
// Gram-Schmidt applied twice, solve the projected real symmetric problem,
// sort by |theta|, test |beta_m s_{m,i}| <= tol |theta_i| from the top, keep
// nconv + (ncv - nconv)/2 Ritz vectors plus the residual direction, restart.
//
// Two basis back ends:
//   host   : basis vectors in host memory, every product goes through
//            laph_matmult with host pointers (the reference's data flow with
//            only the MatShell body on the GPU); orthogonalisation on the host
//            with OpenMP, as SLEPc does with host vectors.
//   device : basis vectors in device memory (SLEPc built with CUDA vectors):
//            products in place on the device, orthogonalisation and restarts
//            with cuBLAS (ZGEMV / ZGEMM), as SLEPc's BV routines do there.
#include <cublas_v2.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "common.cuh"
#include "stencil64.cuh"

namespace laph {
// defined in capi_ctx.cu
int ctx_device_links(laph_ctx* c, const double2** U, int* L, double* lam_l, double* lam_c, int* deg, cudaStream_t* st,
                     int* dev);
}  // namespace laph

using namespace laph;
typedef std::complex<double> cd;

namespace {

// Householder reduction of a real symmetric n x n (row-major) to tridiagonal
// form, accumulating the orthogonal transform in Q: A = Q T Q^T.
void tridiagonalise(int n, std::vector<double>& A, std::vector<double>& d, std::vector<double>& e,
                    std::vector<double>& Q) {
  Q.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) Q[(size_t)i * n + i] = 1.0;
  std::vector<double> v(n), p(n), w(n);
  for (int k = 0; k + 2 < n; ++k) {
    double alpha = 0.0;
    for (int i = k + 1; i < n; ++i) alpha += A[(size_t)i * n + k] * A[(size_t)i * n + k];
    alpha = std::sqrt(alpha);
    if (alpha == 0.0) continue;
    const double x0 = A[(size_t)(k + 1) * n + k];
    if (x0 > 0) alpha = -alpha;
    // v = x - alpha e1, normalised
    double vn = 0.0;
    for (int i = k + 1; i < n; ++i) {
      v[i] = A[(size_t)i * n + k];
      if (i == k + 1) v[i] -= alpha;
      vn += v[i] * v[i];
    }
    vn = std::sqrt(vn);
    if (vn == 0.0) continue;
    for (int i = k + 1; i < n; ++i) v[i] /= vn;
    // A22 <- H A22 H, H = I - 2 v v^T: p = A22 v, q = p - (v.p) v, A22 -= 2(v q^T + q v^T)
    for (int i = k + 1; i < n; ++i) {
      double s = 0.0;
      for (int j = k + 1; j < n; ++j) s += A[(size_t)i * n + j] * v[j];
      p[i] = s;
    }
    double vp = 0.0;
    for (int i = k + 1; i < n; ++i) vp += v[i] * p[i];
    for (int i = k + 1; i < n; ++i) w[i] = p[i] - vp * v[i];
    for (int i = k + 1; i < n; ++i)
      for (int j = k + 1; j < n; ++j) A[(size_t)i * n + j] -= 2.0 * (v[i] * w[j] + w[i] * v[j]);
    A[(size_t)(k + 1) * n + k] = A[(size_t)k * n + k + 1] = alpha;
    for (int i = k + 2; i < n; ++i) A[(size_t)i * n + k] = A[(size_t)k * n + i] = 0.0;
    // Q <- Q H
    for (int r = 0; r < n; ++r) {
      double s = 0.0;
      for (int j = k + 1; j < n; ++j) s += Q[(size_t)r * n + j] * v[j];
      for (int j = k + 1; j < n; ++j) Q[(size_t)r * n + j] -= 2.0 * s * v[j];
    }
  }
  d.resize(n);
  e.assign(n, 0.0);
  for (int i = 0; i < n; ++i) d[i] = A[(size_t)i * n + i];
  for (int i = 0; i + 1 < n; ++i) e[i] = A[(size_t)(i + 1) * n + i];
}

// Implicit QL with Wilkinson shifts on the symmetric tridiagonal (d, e),
// rotating the columns of Z (row-major n x n).  Returns false if an
// eigenvalue needed more than 60 sweeps.
bool tridiag_ql(int n, std::vector<double>& d, std::vector<double>& e, std::vector<double>& Z) {
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    for (;;) {
      int m = l;
      for (; m + 1 < n; ++m) {
        const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) <= 1e-16 * dd) break;
      }
      if (m == l) break;
      if (++iter > 60) return false;
      double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double r = std::hypot(g, 1.0);
      g = d[m] - d[l] + e[l] / (g + (g >= 0 ? r : -r));
      double s = 1.0, c = 1.0, p = 0.0;
      int i = m - 1;
      bool early = false;
      for (; i >= l; --i) {
        double f = s * e[i], b = c * e[i];
        r = std::hypot(f, g);
        e[i + 1] = r;
        if (r == 0.0) {
          d[i + 1] -= p;
          e[m] = 0.0;
          early = true;
          break;
        }
        s = f / r;
        c = g / r;
        g = d[i + 1] - p;
        r = (d[i] - g) * s + 2.0 * c * b;
        p = s * r;
        d[i + 1] = g + p;
        g = c * r - b;
        for (int k = 0; k < n; ++k) {
          const double zf = Z[(size_t)k * n + i + 1];
          Z[(size_t)k * n + i + 1] = s * Z[(size_t)k * n + i] + c * zf;
          Z[(size_t)k * n + i] = c * Z[(size_t)k * n + i] - s * zf;
        }
      }
      if (early) continue;
      d[l] -= p;
      e[l] = g;
      e[m] = 0.0;
    }
  }
  return true;
}

struct SplitMix {
  uint64_t s;
  explicit SplitMix(uint64_t v) : s(v) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  }
  double uniform() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
};

// ---------------------------------------------------------------- bases ----
struct Basis {
  long n = 0;
  int cap = 0;
  virtual ~Basis() {}
  virtual int start(const std::vector<cd>& v0) = 0;              // column 0 = v0
  virtual int op(int j) = 0;                                        // w = T_deg(B) v_j
  virtual int orth(int j, std::vector<cd>& h, double* beta) = 0;  // CGS2 of w on v_0..v_j; v_{j+1} = w/|w|
  virtual int rotate(const std::vector<double>& Zk, int m, int keep) = 0;  // V[:, :keep] = V[:, :m] Zk (m x keep, col-major)
  virtual int copy_col(int from, int to) = 0;
  virtual int fetch(int ncols, double* out) = 0;  // host, column-major complex128
  long long nmatvec = 0;
};

struct HostBasis : Basis {
  laph_ctx* ctx;
  int deg;
  std::vector<cd> V, w, tmp;
  HostBasis(laph_ctx* c, long dim, int m, int dg) : ctx(c), deg(dg) {
    n = dim;
    cap = m + 1;
    V.resize((size_t)dim * cap);
    w.resize(dim);
  }
  cd* col(int j) { return V.data() + (size_t)j * n; }
  int start(const std::vector<cd>& v0) override {
    std::memcpy(static_cast<void*>(col(0)), v0.data(), n * sizeof(cd));
    return LAPH_OK;
  }
  int op(int j) override {
    ++nmatvec;
    return laph_matmult(ctx, reinterpret_cast<const double*>(col(j)), reinterpret_cast<double*>(w.data()), deg, 0);
  }
  int orth(int j, std::vector<cd>& h, double* beta) override {
    std::vector<cd> h2(j + 1);
    for (int pass = 0; pass < 2; ++pass) {
      std::vector<cd>& hh = pass == 0 ? h : h2;
      hh.assign(j + 1, 0.0);
#pragma omp parallel for schedule(static)
      for (int c = 0; c <= j; ++c) {
        cd s = 0.0;
        const cd* vc = col(c);
        for (long i = 0; i < n; ++i) s += std::conj(vc[i]) * w[i];
        hh[c] = s;
      }
#pragma omp parallel for schedule(static)
      for (long i0 = 0; i0 < n; i0 += 512) {
        const long i1 = std::min(n, i0 + 512);
        for (int c = 0; c <= j; ++c) {
          const cd a = hh[c];
          const cd* vc = col(c);
          for (long i = i0; i < i1; ++i) w[i] -= vc[i] * a;
        }
      }
    }
    for (int c = 0; c <= j; ++c) h[c] += h2[c];
    double b = 0.0;
#pragma omp parallel for reduction(+ : b)
    for (long i = 0; i < n; ++i) b += std::norm(w[i]);
    b = std::sqrt(b);
    *beta = b;
    const double ib = 1.0 / b;
    cd* vn = col(j + 1);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) vn[i] = w[i] * ib;
    return LAPH_OK;
  }
  int rotate(const std::vector<double>& Zk, int m, int keep) override {
    tmp.assign((size_t)n * keep, 0.0);
#pragma omp parallel for schedule(static)
    for (long i0 = 0; i0 < n; i0 += 256) {
      const long i1 = std::min(n, i0 + 256);
      for (int c = 0; c < keep; ++c) {
        cd* dst = &tmp[(size_t)c * n];
        for (int r = 0; r < m; ++r) {
          const double z = Zk[(size_t)c * m + r];
          const cd* vr = col(r);
          for (long i = i0; i < i1; ++i) dst[i] += vr[i] * z;
        }
      }
    }
    std::memcpy(static_cast<void*>(V.data()), tmp.data(), (size_t)n * keep * sizeof(cd));
    return LAPH_OK;
  }
  int copy_col(int from, int to) override {
    std::memcpy(static_cast<void*>(col(to)), col(from), n * sizeof(cd));
    return LAPH_OK;
  }
  int fetch(int ncols, double* out) override {
    std::memcpy(out, V.data(), (size_t)n * ncols * sizeof(cd));
    return LAPH_OK;
  }
};

// Basis in host memory whose products call a user callback: what SLEPc's
// EPSSolve does with any MatShell (MatMult -> the registered MATOP_MULT).
struct CallbackBasis : HostBasis {
  int (*mult)(void*, const double*, double*);
  void* user;
  CallbackBasis(long dim, int m, int (*f)(void*, const double*, double*), void* u)
      : HostBasis(nullptr, dim, m, 0), mult(f), user(u) {}
  int op(int j) override {
    ++nmatvec;
    const int rc = mult(user, reinterpret_cast<const double*>(col(j)), reinterpret_cast<double*>(w.data()));
    if (rc != 0) {
      set_error("laph_eps_solve_cb: operator callback returned %d", rc);
      return LAPH_EINVAL;
    }
    return LAPH_OK;
  }
};

#define LAPH_CUBLAS_TRY(expr)                                         \
  do {                                                                \
    cublasStatus_t _s = (expr);                                       \
    if (_s != CUBLAS_STATUS_SUCCESS) {                                \
      set_error("%s:%d: %s failed (%d)", __FILE__, __LINE__, #expr, (int)_s); \
      return LAPH_ECUDA;                                              \
    }                                                                 \
  } while (0)

struct DeviceBasis : Basis {
  laph_ctx* ctx;
  const double2* U = nullptr;
  int L = 0, deg = 0, dev = 0;
  double lam_l = 0, lam_c = 0;
  cudaStream_t st = nullptr;
  cublasHandle_t hb = nullptr;
  double2 *V = nullptr, *w = nullptr, *tmp = nullptr, *h = nullptr, *Zd = nullptr;
  GridBar* bar = nullptr;  // grid barrier of the fused T_deg(B) product
  int* h_err = nullptr;    // page-locked, mapped: set by a barrier that gave up
  int* d_herr = nullptr;
  int ok = 0;
  DeviceBasis(laph_ctx* c, long dim, int m) : ctx(c) {
    n = dim;
    cap = m + 1;
    int dg;
    if (ctx_device_links(ctx, &U, &L, &lam_l, &lam_c, &dg, &st, &dev) != LAPH_OK) return;
    if (cudaMalloc(&V, sizeof(double2) * n * (cap + 1)) != cudaSuccess || cudaMalloc(&w, sizeof(double2) * n) != cudaSuccess ||
        cudaMalloc(&tmp, sizeof(double2) * n * 2) != cudaSuccess || cudaMalloc(&h, sizeof(double2) * 2 * cap) != cudaSuccess ||
        cudaMalloc(&Zd, sizeof(double2) * cap * cap) != cudaSuccess || cudaMalloc(&bar, sizeof(GridBar)) != cudaSuccess ||
        cudaMemset(bar, 0, sizeof(GridBar)) != cudaSuccess ||
        cudaHostAlloc(&h_err, sizeof(int), cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer(reinterpret_cast<void**>(&d_herr), h_err, 0) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    *reinterpret_cast<volatile int*>(h_err) = 0;
    if (cublasCreate(&hb) != CUBLAS_STATUS_SUCCESS) return;
    cublasSetStream(hb, st);
    ok = 1;
  }
  ~DeviceBasis() override {
    if (hb) cublasDestroy(hb);
    cudaFree(V);
    cudaFree(w);
    cudaFree(tmp);
    cudaFree(h);
    cudaFree(Zd);
    cudaFree(bar);
    if (h_err) cudaFreeHost(h_err);
  }
  // nonzero if a grid barrier of any product so far gave up (sticky)
  int barrier_failed() {
    if (cudaStreamSynchronize(st) != cudaSuccess) return 1;
    return *reinterpret_cast<volatile int*>(h_err);
  }
  double2* col(int j) { return V + (size_t)j * n; }
  int start(const std::vector<cd>& v0) override {
    LAPH_CUDA_TRY(cudaMemcpyAsync(col(0), v0.data(), n * sizeof(double2), cudaMemcpyHostToDevice, st));
    return LAPH_OK;
  }
  int op(int j) override {
    ++nmatvec;
    return cheb64_fused(U, L, lam_l, lam_c, deg, col(j), w, tmp, n, bar, d_herr, st);
  }
  int orth(int j, std::vector<cd>& hh, double* beta) override {
    const cuDoubleComplex one = {1.0, 0.0}, zero = {0.0, 0.0}, mone = {-1.0, 0.0};
    cuDoubleComplex* Vc = reinterpret_cast<cuDoubleComplex*>(V);
    cuDoubleComplex* wc = reinterpret_cast<cuDoubleComplex*>(w);
    cuDoubleComplex* hc = reinterpret_cast<cuDoubleComplex*>(h);
    for (int pass = 0; pass < 2; ++pass) {
      LAPH_CUBLAS_TRY(cublasZgemv(hb, CUBLAS_OP_C, (int)n, j + 1, &one, Vc, (int)n, wc, 1, &zero, hc + pass * cap, 1));
      LAPH_CUBLAS_TRY(cublasZgemv(hb, CUBLAS_OP_N, (int)n, j + 1, &mone, Vc, (int)n, hc + pass * cap, 1, &one, wc, 1));
    }
    std::vector<cd> a(2 * cap);
    LAPH_CUDA_TRY(cudaMemcpyAsync(a.data(), h, sizeof(double2) * 2 * cap, cudaMemcpyDeviceToHost, st));
    double nb = 0.0;
    LAPH_CUBLAS_TRY(cublasSetPointerMode(hb, CUBLAS_POINTER_MODE_HOST));
    LAPH_CUBLAS_TRY(cublasDznrm2(hb, (int)n, wc, 1, &nb));  // synchronises
    hh.assign(j + 1, 0.0);
    for (int c = 0; c <= j; ++c) hh[c] = a[c] + a[cap + c];
    *beta = nb;
    const double ib = 1.0 / nb;
    LAPH_CUDA_TRY(cudaMemcpyAsync(col(j + 1), w, n * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    LAPH_CUBLAS_TRY(cublasZdscal(hb, (int)n, &ib, reinterpret_cast<cuDoubleComplex*>(col(j + 1)), 1));
    return LAPH_OK;
  }
  int rotate(const std::vector<double>& Zk, int m, int keep) override {
    std::vector<cd> zc((size_t)m * keep);
    for (size_t i = 0; i < zc.size(); ++i) zc[i] = Zk[i];
    LAPH_CUDA_TRY(cudaMemcpyAsync(Zd, zc.data(), sizeof(double2) * zc.size(), cudaMemcpyHostToDevice, st));
    const cuDoubleComplex one = {1.0, 0.0}, zero = {0.0, 0.0};
    // out-of-place into column block [cap - keep ... ) is not available; use tmp columns in chunks of 2
    double2* out = nullptr;
    if (cudaMalloc(&out, sizeof(double2) * n * keep) != cudaSuccess) {
      cudaGetLastError();
      set_error("krylov-schur restart: allocation failed");
      return LAPH_ENOMEM;
    }
    LAPH_CUBLAS_TRY(cublasZgemm(hb, CUBLAS_OP_N, CUBLAS_OP_N, (int)n, keep, m, &one, reinterpret_cast<cuDoubleComplex*>(V),
                                (int)n, reinterpret_cast<cuDoubleComplex*>(Zd), m, &zero,
                                reinterpret_cast<cuDoubleComplex*>(out), (int)n));
    LAPH_CUDA_TRY(cudaMemcpyAsync(V, out, sizeof(double2) * n * keep, cudaMemcpyDeviceToDevice, st));
    LAPH_CUDA_TRY(cudaStreamSynchronize(st));
    cudaFree(out);
    return LAPH_OK;
  }
  int copy_col(int from, int to) override {
    LAPH_CUDA_TRY(cudaMemcpyAsync(col(to), col(from), n * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    return LAPH_OK;
  }
  int fetch(int ncols, double* out) override {
    LAPH_CUDA_TRY(cudaMemcpyAsync(out, V, sizeof(double2) * n * ncols, cudaMemcpyDeviceToHost, st));
    LAPH_CUDA_TRY(cudaStreamSynchronize(st));
    return LAPH_OK;
  }
};

}  // namespace

static int krylov_schur(Basis* B, long dim, int nev, int m, double tol, int max_it, uint64_t seed, double* theta_out,
                        double* V_out, int* nconv_out, int* its_out, long long* nmatvec_out) {
  int rc = LAPH_OK;
  {
    SplitMix rng(seed);
    std::vector<cd> v0(dim);
    double nrm = 0.0;
    for (long i = 0; i < dim; ++i) {
      const double u1 = rng.uniform(), u2 = rng.uniform();
      const double r = std::sqrt(-2.0 * std::log(u1));
      v0[i] = cd(r * std::cos(2 * M_PI * u2), r * std::sin(2 * M_PI * u2));
      nrm += std::norm(v0[i]);
    }
    nrm = 1.0 / std::sqrt(nrm);
    for (auto& x : v0) x *= nrm;
    rc = B->start(v0);
  }
  std::vector<double> T((size_t)m * m, 0.0), A, d, e, Z;
  std::vector<int> ord(m);
  std::vector<cd> h;
  int k = 0, nconv = 0, it = 0;
  double beta_m = 0.0;
  bool done = false;
  for (it = 1; rc == LAPH_OK && it <= max_it; ++it) {
    for (int j = k; j < m && rc == LAPH_OK; ++j) {
      rc = B->op(j);
      if (rc != LAPH_OK) break;
      double beta;
      rc = B->orth(j, h, &beta);
      T[(size_t)j * m + j] = h[j].real();
      if (j + 1 < m) T[(size_t)j * m + j + 1] = T[(size_t)(j + 1) * m + j] = beta;
      beta_m = beta;
    }
    if (rc != LAPH_OK) break;
    A = T;
    tridiagonalise(m, A, d, e, Z);
    if (!tridiag_ql(m, d, e, Z)) {
      set_error("laph_eps_solve: projected eigenproblem did not converge");
      rc = LAPH_ENOTCONV;
      break;
    }
    for (int i = 0; i < m; ++i) ord[i] = i;
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return std::fabs(d[a]) > std::fabs(d[b]); });
    int nc = 0;
    for (int i = 0; i < m; ++i) {
      const double res = std::fabs(beta_m * Z[(size_t)(m - 1) * m + ord[i]]);
      if (res <= tol * std::fabs(d[ord[i]])) ++nc;
      else break;
    }
    nconv = nc;
    done = nconv >= nev || it == max_it;
    int keep = done ? nev : nconv + std::max(1, (m - nconv) / 2);
    if (!done && keep > m - 1) keep = m - 1;
    std::vector<double> Zk((size_t)m * keep);
    for (int c = 0; c < keep; ++c)
      for (int r = 0; r < m; ++r) Zk[(size_t)c * m + r] = Z[(size_t)r * m + ord[c]];
    if (done) {
      rc = B->rotate(Zk, m, keep);
      for (int c = 0; c < nev; ++c) theta_out[c] = d[ord[c]];
      if (rc == LAPH_OK && V_out) rc = B->fetch(nev, V_out);
      break;
    }
    rc = B->rotate(Zk, m, keep);                   // Ritz vectors into columns [0, keep)
    if (rc == LAPH_OK) rc = B->copy_col(m, keep);  // then the residual direction v_m -> v_keep
    std::fill(T.begin(), T.end(), 0.0);
    for (int c = 0; c < keep; ++c) {
      T[(size_t)c * m + c] = d[ord[c]];
      const double b = beta_m * Z[(size_t)(m - 1) * m + ord[c]];
      T[(size_t)c * m + keep] = T[(size_t)keep * m + c] = b;
    }
    k = keep;
  }
  if (nconv_out) *nconv_out = nconv;
  if (its_out) *its_out = std::min(it, max_it);
  if (nmatvec_out) *nmatvec_out = B->nmatvec;
  if (rc != LAPH_OK) return rc;
  if (nconv < nev) {
    set_error("laph_eps_solve: %d of %d pairs converged after %d restarts", nconv, nev, max_it);
    return LAPH_ENOTCONV;
  }
  return LAPH_OK;
}

static int ncv_default(int nev, int ncv, long dim) {
  if (ncv <= 0) ncv = std::max(2 * nev, nev + 15);
  if (ncv > dim - 1) ncv = (int)dim - 1;
  return ncv;
}

extern "C" int laph_eps_solve(laph_ctx* ctx, int nev, int ncv, double tol, int max_it, int device_basis, uint64_t seed,
                              double* theta_out, double* V_out, int* nconv_out, int* its_out, long long* nmatvec_out) {
  const double2* U;
  int L, deg, dev;
  double lam_l, lam_c;
  cudaStream_t st;
  LAPH_TRY(ctx_device_links(ctx, &U, &L, &lam_l, &lam_c, &deg, &st, &dev));
  const long dim = 3L * L * L * L;
  if (nev < 1 || !theta_out || !(tol > 0.0) || max_it < 1 || deg < 1) {
    set_error("laph_eps_solve: bad argument");
    return LAPH_EINVAL;
  }
  const int m = ncv_default(nev, ncv, dim);
  if (nev >= m) {
    set_error("laph_eps_solve: nev %d too large for dim %ld", nev, dim);
    return LAPH_EINVAL;
  }
  Basis* B = nullptr;
  if (device_basis) {
    auto* db = new DeviceBasis(ctx, dim, m);
    db->deg = deg;
    if (!db->ok) {
      delete db;
      set_error("laph_eps_solve: device basis allocation failed");
      return LAPH_ENOMEM;
    }
    B = db;
  } else {
    B = new HostBasis(ctx, dim, m, deg);
  }
  int rc = krylov_schur(B, dim, nev, m, tol, max_it, seed, theta_out, V_out, nconv_out, its_out, nmatvec_out);
  if (device_basis && static_cast<DeviceBasis*>(B)->barrier_failed()) {
    set_error("laph_eps_solve: a grid barrier of the fused product gave up waiting; the result is not valid");
    rc = LAPH_ECUDA;
  }
  delete B;
  return rc;
}

extern "C" int laph_eps_solve_cb(long long dim, int (*mult)(void* user, const double* x, double* y), void* user, int nev,
                                 int ncv, double tol, int max_it, uint64_t seed, double* theta_out, double* V_out,
                                 int* nconv_out, int* its_out, long long* nmatvec_out) {
  if (dim < 2 || !mult || nev < 1 || !theta_out || !(tol > 0.0) || max_it < 1) {
    set_error("laph_eps_solve_cb: bad argument");
    return LAPH_EINVAL;
  }
  const int m = ncv_default(nev, ncv, (long)dim);
  if (nev >= m) {
    set_error("laph_eps_solve_cb: nev %d too large for dim %lld", nev, dim);
    return LAPH_EINVAL;
  }
  CallbackBasis B((long)dim, m, mult, user);
  return krylov_schur(&B, (long)dim, nev, m, tol, max_it, seed, theta_out, V_out, nconv_out, its_out, nmatvec_out);
}
