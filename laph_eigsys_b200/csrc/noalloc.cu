// noalloc.cu -- laph_matmult_noalloc: the FP64 MatShell product
// y = T_deg(B) x for callers that must not allocate device memory.
//
// Who needs it: callers that cannot call cudaMalloc at the point where they
// need the product -- a host framework that owns the whole device memory
// budget through its own pool and forbids other allocations, a long-running
// service that allocates only at start-up, or a real-time loop that cannot
// afford the implicit synchronisation of cudaMalloc / cudaFree.  Such a
// caller owns its links, x and y on the device and only needs somewhere to
// keep the two Chebyshev temporaries of tv_iter
// (modules/shell_matop.cpp:136-168).
//
// Those temporaries live in g_noalloc_scratch below: a file-scope device
// array sized for timeslices up to kNoAllocMaxL^3 (3 MiB).  Every GPU that
// loads this library keeps that array until the process exits.  Host code
// cannot pass g_noalloc_scratch to a kernel directly (on the host the name is
// only a stand-in, not a device address), so the first call in each CUDA
// context looks the address up with cudaGetSymbolAddress while that context
// is current, checks it, and caches it under the context's unique ID
// (cuCtxGetId: never reused in a process, so a context created after
// cudaDeviceReset or cuCtxDestroy gets a fresh lookup).  Make that first call
// before any stream capture begins.
//
// Every call shares the one array and it keeps the previous call's contents.
// Nothing in it has to start at zero: each Chebyshev step writes every
// element of its output before any later step reads it.  Calls whose work
// overlaps on the GPU (different streams, or different host threads, on the
// same device) race on the array; serialise them on one stream.
#include <cuda.h>

#include <mutex>
#include <utility>
#include <vector>

#include "common.cuh"

namespace laph {

constexpr int kNoAllocMaxL = 32;
constexpr size_t kNoAllocMaxDim = 3ull * kNoAllocMaxL * kNoAllocMaxL * kNoAllocMaxL;

static __device__ __align__(256) double2 g_noalloc_scratch[2 * kNoAllocMaxDim];

namespace {
using CtxGetCurrent = CUresult (*)(CUcontext*);
using CtxGetId = CUresult (*)(CUcontext, unsigned long long*);

std::mutex g_noalloc_mu;
std::vector<std::pair<unsigned long long, double2*>> g_noalloc_ptr;  // (context ID, scratch address)
CtxGetCurrent g_get_current = nullptr;
CtxGetId g_get_id = nullptr;

// Unique ID of the calling thread's current context (0: none current).
int current_ctx_id(unsigned long long* id) {
  *id = 0;
  CUcontext c = nullptr;
  if (g_get_current(&c) != CUDA_SUCCESS) {
    set_error("laph_matmult_noalloc: cuCtxGetCurrent failed");
    return LAPH_ECUDA;
  }
  if (c && g_get_id(c, id) != CUDA_SUCCESS) {
    set_error("laph_matmult_noalloc: cuCtxGetId failed");
    return LAPH_ECUDA;
  }
  return LAPH_OK;
}

int noalloc_scratch(double2** out) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_get_current || !g_get_id) {
    void *f1 = nullptr, *f2 = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 12000, cudaEnableDefault, &q1) != cudaSuccess ||
        cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000, cudaEnableDefault, &q2) != cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2) {
      cudaGetLastError();
      set_error("laph_matmult_noalloc: the driver does not provide cuCtxGetCurrent / cuCtxGetId");
      return LAPH_ECUDA;
    }
    g_get_current = reinterpret_cast<CtxGetCurrent>(f1);
    g_get_id = reinterpret_cast<CtxGetId>(f2);
  }
  unsigned long long id = 0;
  LAPH_TRY(current_ctx_id(&id));
  if (id != 0)
    for (const auto& e : g_noalloc_ptr)
      if (e.first == id) {
        *out = e.second;
        return LAPH_OK;
      }
  // first call in this context: resolve the array's device address (this also
  // makes the device's primary context current if no context was)
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || p == nullptr) {
    cudaGetLastError();
    set_error("laph_matmult_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
    return LAPH_ECUDA;
  }
  LAPH_TRY(current_ctx_id(&id));
  if (id == 0) {
    set_error("laph_matmult_noalloc: no CUDA context is current");
    return LAPH_ECUDA;
  }
  g_noalloc_ptr.emplace_back(id, static_cast<double2*>(p));
  *out = static_cast<double2*>(p);
  return LAPH_OK;
}
}  // namespace

// y = c_hop * hop(x) + c_diag * x + c_z * z, links in the boundary layout
// LAPH_LAYOUT_ROWMAJOR: U[((site*3 + mu)*9 + 3a + b)] (complex128).
template <bool HAS_Z>
__global__ void __launch_bounds__(128) k_hop64_rowmajor(const double2* __restrict__ U, Lat g,
                                                        const double2* __restrict__ x, const double2* __restrict__ z,
                                                        double2* __restrict__ y, double c_hop, double c_diag,
                                                        double c_z) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V3) return;
  int sx, sy, sz;
  site_xyz(g, s, sx, sy, sz);
  double2 acc[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
#pragma unroll
  for (int mu = 0; mu < 3; ++mu) {
    const int up = nb_up(g, sx, sy, sz, mu), dn = nb_dn(g, sx, sy, sz, mu);
    const double2* uf = U + ((size_t)s * 3 + mu) * 9;
    const double2* ub = U + ((size_t)dn * 3 + mu) * 9;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        cfma(acc[a], __ldg(uf + 3 * a + b), __ldg(x + 3 * (size_t)up + b));
        cfmac(acc[a], __ldg(ub + 3 * b + a), __ldg(x + 3 * (size_t)dn + b));
      }
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double2 xs = __ldg(x + 3 * (size_t)s + a);
    double2 r = make_double2(c_hop * acc[a].x + c_diag * xs.x, c_hop * acc[a].y + c_diag * xs.y);
    if (HAS_Z) {
      const double2 zz = __ldg(z + 3 * (size_t)s + a);
      r.x += c_z * zz.x;
      r.y += c_z * zz.y;
    }
    y[3 * (size_t)s + a] = r;
  }
}

}  // namespace laph

using namespace laph;

extern "C" int laph_matmult_noalloc(const double* links, int L, double lam_l, double lam_c, int deg, const double* x,
                                    double* y, void* stream) {
  if (!links || !x || !y) {
    set_error("laph_matmult_noalloc: null pointer");
    return LAPH_EINVAL;
  }
  if (L < 3 || L > kNoAllocMaxL) {
    set_error("laph_matmult_noalloc: L = %d is outside [3, %d], the size its fixed %zu-byte scratch array holds", L,
              kNoAllocMaxL, sizeof(double2) * 2 * kNoAllocMaxDim);
    return LAPH_EINVAL;
  }
  if (deg < 1 || !(lam_l > lam_c)) {
    set_error("laph_matmult_noalloc: need deg >= 1 and lam_l > lam_c");
    return LAPH_EINVAL;
  }
  const size_t vbytes = sizeof(double2) * 3 * (size_t)L * L * L;
  if (ranges_overlap(x, y, vbytes)) {
    set_error("laph_matmult_noalloc: x and y overlap (the product reads x while it writes y)");
    return LAPH_EINVAL;
  }
  double2* scratch = nullptr;
  LAPH_TRY(noalloc_scratch(&scratch));
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  const Lat g = make_lat(L);
  const size_t dim = 3 * (size_t)g.V3;
  const double c = 2.0 / (lam_l - lam_c);
  const double a = 1.0 + c * lam_c;
  const double2* U = reinterpret_cast<const double2*>(links);
  const double2* dx = reinterpret_cast<const double2*>(x);
  double2* dy = reinterpret_cast<double2*>(y);
  const dim3 grid(ceil_div(g.V3, 128));
  if (deg == 1) {
    k_hop64_rowmajor<false><<<grid, 128, 0, st>>>(U, g, dx, nullptr, dy, c, a - 6.0 * c, 0.0);
    LAPH_CUDA_TRY(cudaGetLastError());
    return LAPH_OK;
  }
  // T_n in bufs[idx(n)] with idx(deg) = y: three consecutive T's never share a buffer
  double2* bufs[3] = {scratch, scratch + dim, dy};
  auto idx = [deg](int n) { return (((2 - (deg - n)) % 3) + 3) % 3; };
  k_hop64_rowmajor<false><<<grid, 128, 0, st>>>(U, g, dx, nullptr, bufs[idx(1)], c, a - 6.0 * c, 0.0);
  for (int n = 2; n <= deg; ++n) {
    const double2* prev = (n == 2) ? dx : bufs[idx(n - 2)];
    k_hop64_rowmajor<true><<<grid, 128, 0, st>>>(U, g, bufs[idx(n - 1)], prev, bufs[idx(n)], 2.0 * c,
                                                 2.0 * (a - 6.0 * c), -1.0);
  }
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}
