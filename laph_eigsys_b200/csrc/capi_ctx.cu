// capi_ctx.cu -- single-timeslice context of the C ABI: the device-resident
// replacement for the IO/Nav/Tslice singletons that MatMult_Laplacian2D reads
// (modules/shell_matop.cpp:9-11), plus the FP64 MatMult body and smearing.
#include <cstring>
#include <vector>

#include "common.cuh"
#include "links.cuh"
#include "smear.cuh"
#include "stencil64.cuh"

struct laph_ctx {
  int dev = 0;
  laph::Lat g{};
  double lam_l = 0, lam_c = 0;
  int deg = 0;
  cudaStream_t st = nullptr;
  double2* U = nullptr;     // [3][9][V3] site-minor
  double2* Utmp = nullptr;  // smearing output
  double2* dec = nullptr;   // HYP decorated links [6][9][V3]
  double2* vec = nullptr;   // 4 vectors of dim: x, y, tmp0, tmp1
  double2* h_stage = nullptr;  // pinned staging, 2 vectors
  double* d_scalar = nullptr;
  laph::GridBar* bar = nullptr;  // grid barrier of the fused MatMult
  int* h_err = nullptr;          // page-locked, mapped: set by a grid barrier that gave up
  int* d_herr = nullptr;         // its device address
};

using namespace laph;

namespace laph {
// Device view of a context for the in-library Krylov-Schur driver.
int ctx_device_links(laph_ctx* c, const double2** U, int* L, double* lam_l, double* lam_c, int* deg, cudaStream_t* st,
                     int* dev) {
  if (!c) {
    set_error("null context");
    return LAPH_EINVAL;
  }
  LAPH_CUDA_TRY(cudaSetDevice(c->dev));
  *U = c->U;
  *L = c->g.L;
  *lam_l = c->lam_l;
  *lam_c = c->lam_c;
  *deg = c->deg;
  *st = c->st;
  *dev = c->dev;
  return LAPH_OK;
}
}  // namespace laph

namespace {
int ctx_check(laph_ctx* c) {
  if (!c) {
    set_error("null context");
    return LAPH_EINVAL;
  }
  LAPH_CUDA_TRY(cudaSetDevice(c->dev));
  return LAPH_OK;
}
}  // namespace

extern "C" {

int laph_ctx_create(laph_ctx** out, const laph_params* p) {
  if (!out || !p || p->L < 3 || p->L > 512) {
    set_error("laph_ctx_create: bad argument (L must be in [3, 512])");
    return LAPH_EINVAL;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("laph_ctx_create: no CUDA device");
    return LAPH_ENODEV;
  }
  if (p->device < 0 || p->device >= ndev) {
    set_error("laph_ctx_create: device %d out of range", p->device);
    return LAPH_EINVAL;
  }
  laph_ctx* c = new laph_ctx();
  c->dev = p->device;
  c->g = make_lat(p->L);
  c->lam_l = p->lam_l;
  c->lam_c = p->lam_c;
  c->deg = p->deg;
  auto fail = [&](int s) {
    laph_ctx_destroy(c);
    return s;
  };
  if (cudaSetDevice(c->dev) != cudaSuccess) return fail(LAPH_ECUDA);
  const size_t V3 = c->g.V3, dim = 3 * V3;
  if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&c->U, sizeof(double2) * 27 * V3) != cudaSuccess ||
      cudaMalloc(&c->Utmp, sizeof(double2) * 27 * V3) != cudaSuccess ||
      cudaMalloc(&c->dec, sizeof(double2) * 54 * V3) != cudaSuccess ||
      cudaMalloc(&c->vec, sizeof(double2) * 4 * dim) != cudaSuccess ||
      cudaMalloc(&c->d_scalar, sizeof(double) * 64) != cudaSuccess ||
      cudaMalloc(&c->bar, sizeof(GridBar)) != cudaSuccess || cudaMemset(c->bar, 0, sizeof(GridBar)) != cudaSuccess ||
      cudaHostAlloc(&c->h_err, sizeof(int), cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer(reinterpret_cast<void**>(&c->d_herr), c->h_err, 0) != cudaSuccess ||
      cudaMallocHost(&c->h_stage, sizeof(double2) * 2 * dim) != cudaSuccess) {
    cudaGetLastError();
    set_error("laph_ctx_create: allocation failed for L=%d", p->L);
    return fail(LAPH_ENOMEM);
  }
  // identity links, as Tslice::init (timeslice.cpp:19-31)
  std::vector<double2> id(27 * V3, make_double2(0.0, 0.0));
  for (int d = 0; d < 3; ++d)
    for (int a = 0; a < 3; ++a)
      for (size_t s = 0; s < V3; ++s) id[(size_t)(d * 9 + 4 * a) * V3 + s].x = 1.0;
  if (cudaMemcpy(c->U, id.data(), sizeof(double2) * 27 * V3, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    return fail(LAPH_ECUDA);
  }
  *out = c;
  return LAPH_OK;
}

int laph_ctx_destroy(laph_ctx* c) {
  if (!c) return LAPH_OK;
  cudaSetDevice(c->dev);
  if (c->st) cudaStreamSynchronize(c->st);
  cudaFree(c->U);
  cudaFree(c->Utmp);
  cudaFree(c->dec);
  cudaFree(c->vec);
  cudaFree(c->d_scalar);
  cudaFree(c->bar);
  if (c->h_err) cudaFreeHost(c->h_err);
  if (c->h_stage) cudaFreeHost(c->h_stage);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
  return LAPH_OK;
}

int laph_ctx_stream(laph_ctx* c, void** stream) {
  if (!c || !stream) {
    set_error("laph_ctx_stream: bad argument");
    return LAPH_EINVAL;
  }
  *stream = static_cast<void*>(c->st);
  return LAPH_OK;
}

int laph_ctx_set_window(laph_ctx* c, double lam_l, double lam_c, int deg) {
  LAPH_TRY(ctx_check(c));
  if (!(lam_l > lam_c)) {
    set_error("laph_ctx_set_window: need lam_l > lam_c");
    return LAPH_EINVAL;
  }
  c->lam_l = lam_l;
  c->lam_c = lam_c;
  c->deg = deg;
  return LAPH_OK;
}

int laph_set_links(laph_ctx* c, const double* links, int layout) {
  LAPH_TRY(ctx_check(c));
  if (!links) {
    set_error("laph_set_links: null links");
    return LAPH_EINVAL;
  }
  const int V3 = c->g.V3;
  LAPH_TRY(check_links_finite(links, layout, V3, "laph_set_links"));
  std::vector<double2> soa(27 * (size_t)V3);
  LAPH_TRY(links_to_soa(links, layout, V3, soa.data()));
  LAPH_CUDA_TRY(cudaMemcpyAsync(c->U, soa.data(), sizeof(double2) * soa.size(), cudaMemcpyHostToDevice, c->st));
  LAPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  return LAPH_OK;
}

int laph_get_links(laph_ctx* c, double* links, int layout) {
  LAPH_TRY(ctx_check(c));
  if (!links) {
    set_error("laph_get_links: null links");
    return LAPH_EINVAL;
  }
  const int V3 = c->g.V3;
  std::vector<double2> soa(27 * (size_t)V3);
  LAPH_CUDA_TRY(cudaMemcpyAsync(soa.data(), c->U, sizeof(double2) * soa.size(), cudaMemcpyDeviceToHost, c->st));
  LAPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  return soa_to_links(soa.data(), V3, layout, links);
}

int laph_smear(laph_ctx* c, int kind, double p1, double p2, int iters, int compat) {
  LAPH_TRY(ctx_check(c));
  if (iters < 0) {
    set_error("laph_smear: negative iteration count");
    return LAPH_EINVAL;
  }
  LAPH_TRY(smear_batch(c->U, c->Utmp, c->dec, c->g.L, 1, kind, p1, p2, iters, compat, c->st));
  LAPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  return LAPH_OK;
}

static int stage_in(laph_ctx* c, const double* x, int on_device, const double2** dx) {
  const size_t dim = 3 * (size_t)c->g.V3;
  if (on_device) {
    *dx = reinterpret_cast<const double2*>(x);
    return LAPH_OK;
  }
  std::memcpy(c->h_stage, x, sizeof(double2) * dim);
  LAPH_CUDA_TRY(cudaMemcpyAsync(c->vec, c->h_stage, sizeof(double2) * dim, cudaMemcpyHostToDevice, c->st));
  *dx = c->vec;
  return LAPH_OK;
}

static int stage_out(laph_ctx* c, double* y, int on_device) {
  if (on_device) {
    LAPH_CUDA_TRY(cudaStreamSynchronize(c->st));
    return LAPH_OK;
  }
  const size_t dim = 3 * (size_t)c->g.V3;
  LAPH_CUDA_TRY(cudaMemcpyAsync(c->h_stage + dim, c->vec + dim, sizeof(double2) * dim, cudaMemcpyDeviceToHost, c->st));
  LAPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  std::memcpy(y, c->h_stage + dim, sizeof(double2) * dim);
  return LAPH_OK;
}

int laph_matmult(laph_ctx* c, const double* x, double* y, int deg, int on_device) {
  LAPH_TRY(ctx_check(c));
  if (!x || !y || deg < 1) {
    set_error("laph_matmult: bad argument (deg must be >= 1)");
    return LAPH_EINVAL;
  }
  if (!(c->lam_l > c->lam_c)) {
    set_error("laph_matmult: window needs lam_l > lam_c");
    return LAPH_EINVAL;
  }
  const size_t dim = 3 * (size_t)c->g.V3;
  if (on_device && ranges_overlap(x, y, sizeof(double2) * dim)) {
    set_error("laph_matmult: x and y overlap (the product reads x while it writes y)");
    return LAPH_EINVAL;
  }
  const double2* dx;
  LAPH_TRY(stage_in(c, x, on_device, &dx));
  double2* dy = on_device ? reinterpret_cast<double2*>(y) : c->vec + dim;
  // the whole recurrence in one launch (tv_iter, shell_matop.cpp:136-168)
  *reinterpret_cast<volatile int*>(c->h_err) = 0;
  LAPH_TRY(cheb64_fused(c->U, c->g.L, c->lam_l, c->lam_c, deg, dx, dy, c->vec + 2 * dim, dim, c->bar, c->d_herr,
                        c->st));
  LAPH_TRY(stage_out(c, y, on_device));  // synchronises the stream
  if (*reinterpret_cast<volatile int*>(c->h_err)) {
    cudaMemsetAsync(c->bar, 0, sizeof(GridBar), c->st);
    cudaStreamSynchronize(c->st);
    *reinterpret_cast<volatile int*>(c->h_err) = 0;
    set_error("laph_matmult: a grid barrier of the fused product gave up waiting; y is not valid");
    return LAPH_ECUDA;
  }
  return LAPH_OK;
}

int laph_apply_neglap(laph_ctx* c, const double* x, double* y, int on_device) {
  LAPH_TRY(ctx_check(c));
  if (!x || !y) {
    set_error("laph_apply_neglap: null vector");
    return LAPH_EINVAL;
  }
  const size_t dim = 3 * (size_t)c->g.V3;
  if (on_device && ranges_overlap(x, y, sizeof(double2) * dim)) {
    set_error("laph_apply_neglap: x and y overlap (the stencil reads x while it writes y)");
    return LAPH_EINVAL;
  }
  const double2* dx;
  LAPH_TRY(stage_in(c, x, on_device, &dx));
  double2* dy = on_device ? reinterpret_cast<double2*>(y) : c->vec + dim;
  LAPH_TRY(hop64(c->U, c->g.L, dx, nullptr, dy, dim, 1, -1.0, 6.0, 0.0, c->st));
  return stage_out(c, y, on_device);
}

int laph_get_diagonal(laph_ctx* c, double* diag, int on_device) {
  LAPH_TRY(ctx_check(c));
  const size_t dim = 3 * (size_t)c->g.V3;
  std::vector<double2> h(dim, make_double2(-6.0, 0.0));
  if (on_device) {
    LAPH_CUDA_TRY(cudaMemcpyAsync(diag, h.data(), sizeof(double2) * dim, cudaMemcpyHostToDevice, c->st));
    LAPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  } else {
    std::memcpy(diag, h.data(), sizeof(double2) * dim);
  }
  return LAPH_OK;
}

int laph_plaquette(laph_ctx* c, double* plaq) {
  LAPH_TRY(ctx_check(c));
  LAPH_TRY(plaquette_batch(c->U, c->g.L, 1, c->d_scalar, c->st));
  LAPH_CUDA_TRY(cudaMemcpyAsync(plaq, c->d_scalar, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  LAPH_CUDA_TRY(cudaStreamSynchronize(c->st));
  return LAPH_OK;
}

}  // extern "C"
