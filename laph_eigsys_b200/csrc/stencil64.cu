// stencil64.cu -- FP64 covariant-Laplacian stencils.
//
// One kernel covers the reference's tv2 (modules/shell_matop.cpp:16-103) and
// one step of tv_iter's Chebyshev recurrence (:136-168):
//     y = c_hop * hop(x) + c_diag * x + c_z * z,
//     hop(x)(s) = sum_mu U_mu(s) x(s+mu) + U_mu(s-mu)^dag x(s-mu),
// so  B x          : c_hop = c,  c_diag = a - 6c, c_z = 0
//     2 B x - z    : c_hop = 2c, c_diag = 2(a-6c), c_z = -1
//     (-Delta) x   : c_hop = -1, c_diag = 6.
// Vectors keep the reference layout (complex128, index 3*site + colour); a
// block of ncol vectors is column-major with column stride ld.  One thread per
// (site, column); consecutive threads take consecutive sites so every
// 48-byte site vector and every link element is read coalesced.
#include <algorithm>
#include <mutex>

#include "stencil64.cuh"
#include "su3.cuh"

namespace laph {

template <bool HAS_Z>
__global__ void __launch_bounds__(128) k_hop64(const double2* __restrict__ U, Lat g, const double2* __restrict__ X,
                                               const double2* __restrict__ Z, double2* __restrict__ Y, size_t ld,
                                               double c_hop, double c_diag, double c_z) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V3) return;
  const size_t col = (size_t)blockIdx.y * ld;
  const double2* x = X + col;
  int sx, sy, sz;
  site_xyz(g, s, sx, sy, sz);
  double2 acc[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
#pragma unroll
  for (int mu = 0; mu < 3; ++mu) {
    const int up = nb_up(g, sx, sy, sz, mu);
    const int dn = nb_dn(g, sx, sy, sz, mu);
    double2 xu[3], xd[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      xu[b] = __ldg(x + 3 * (size_t)up + b);
      xd[b] = __ldg(x + 3 * (size_t)dn + b);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        cfma(acc[a], __ldg(U + (size_t)(mu * 9 + 3 * a + b) * g.V3 + s), xu[b]);
        cfmac(acc[a], __ldg(U + (size_t)(mu * 9 + 3 * b + a) * g.V3 + dn), xd[b]);
      }
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double2 xs = __ldg(x + 3 * (size_t)s + a);
    double2 r = make_double2(c_hop * acc[a].x + c_diag * xs.x, c_hop * acc[a].y + c_diag * xs.y);
    if (HAS_Z) {
      const double2 zz = __ldg(Z + col + 3 * (size_t)s + a);
      r.x += c_z * zz.x;
      r.y += c_z * zz.y;
    }
    Y[col + 3 * (size_t)s + a] = r;
  }
}

int hop64(const double2* U, int L, const double2* X, const double2* Z, double2* Y, size_t ld, int ncol, double c_hop,
          double c_diag, double c_z, cudaStream_t st) {
  const Lat g = make_lat(L);
  const dim3 grid(ceil_div(g.V3, 128), ncol);
  if (Z)
    k_hop64<true><<<grid, 128, 0, st>>>(U, g, X, Z, Y, ld, c_hop, c_diag, c_z);
  else
    k_hop64<false><<<grid, 128, 0, st>>>(U, g, X, nullptr, Y, ld, c_hop, c_diag, 0.0);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}

// y = T_deg(B) x, B = c(hop - 6) + a (tv_iter, shell_matop.cpp:136-168).
// tmp must hold 2 vectors of dim = 3*V3 (column stride ld).
int cheb64(const double2* U, int L, double lam_l, double lam_c, int deg, const double2* x, double2* y, double2* tmp,
           size_t ld, int ncol, cudaStream_t st) {
  const double c = 2.0 / (lam_l - lam_c);
  const double a = 1.0 + c * lam_c;
  if (deg <= 1) return hop64(U, L, x, nullptr, y, ld, ncol, c, a - 6.0 * c, 0.0, st);
  // T_n lives in bufs[idx(n)], idx(n) = (2 - (deg - n)) mod 3, so T_deg lands
  // in y and three consecutive T's never share a buffer.
  double2* bufs[3] = {tmp, tmp + ld * ncol, y};
  auto idx = [deg](int n) { return (((2 - (deg - n)) % 3) + 3) % 3; };
  LAPH_TRY(hop64(U, L, x, nullptr, bufs[idx(1)], ld, ncol, c, a - 6.0 * c, 0.0, st));
  for (int n = 2; n <= deg; ++n) {
    const double2* prev = (n == 2) ? x : bufs[idx(n - 2)];
    LAPH_TRY(hop64(U, L, bufs[idx(n - 1)], prev, bufs[idx(n)], ld, ncol, 2.0 * c, 2.0 * (a - 6.0 * c), -1.0, st));
  }
  return LAPH_OK;
}


// ------------------------------------------- fused T_deg(B) x, one launch ---
// The plain form's MatMult in ONE cooperative launch: every thread keeps its
// site for the whole recurrence, so the links are read from HBM once per
// product (forward links in 108 registers, backward links U_mu(s - mu) in
// shared memory, as the block stencils keep them) instead of once per step,
// and the deg steps are separated by a grid barrier instead of kernel
// boundaries.  At 32^3 the whole product (links 14 MB, three vectors of
// 1.5 MB) then runs from L2.  The T_n written inside the launch are read
// with ld.global.cg (L2, never a stale L1 line); only x, read-only for the
// launch, goes through the non-coherent path.  Used when one site per thread
// fits the device's co-resident CTAs (up to 296 CTAs of 128 sites on a
// B200: L <= 33); otherwise a grid-stride variant reads the links per step.

// Grid barrier with a bounded wait, one atomic per CTA and arrival: every CTA
// adds 1 to the counter except CTA 0, which adds 2^31 - (nblk - 1), so the
// last arrival flips bit 31 and leaves the low bits at zero for the next
// barrier; a CTA waits for bit 31 to differ from the value its own add
// returned (no reset, no second word).  The add is a release and the polling
// load an acquire at GPU scope; with the CTA barriers on either side they order
// every thread's step-n writes before every thread's step-n+1 reads.  A CTA that waits longer than
// kBarSpinLimit polls sets `err` (and *herr, page-locked host memory the host
// reads after its synchronisation) and every CTA leaves at its next barrier.
// Cooperative launches guarantee co-residency, so the limit is a safety net.
constexpr unsigned kBarSpinLimit = 1u << 24;

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ bool grid_barrier(GridBar* b, unsigned nblk, int* herr) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned inc = blockIdx.x == 0 ? 0x80000000u - (nblk - 1) : 1u;
    // release: the CTA's writes (ordered before this thread by the CTA barrier
    // above) become visible to every CTA whose acquire load sees this arrival
    unsigned old;
    asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(&b->count), "r"(inc) : "memory");
    bool ok = true;
    unsigned it = 0;
    while (((ld_acquire_gpu(&b->count) ^ old) & 0x80000000u) == 0) {
      if ((++it & 1023u) == 0 && (it > kBarSpinLimit || *reinterpret_cast<volatile int*>(&b->err))) {
        atomicExch(&b->err, 1);
        *reinterpret_cast<volatile int*>(herr) = 1;
        ok = false;
        break;
      }
    }
    s_ok = ok && *reinterpret_cast<volatile int*>(&b->err) == 0;
  }
  __syncthreads();
  return s_ok != 0;
}

constexpr int kFusedSmem = 27 * 128 * (int)sizeof(double2);

template <bool RESIDENT>
__global__ void __launch_bounds__(128, 2)
    k_cheb64_fused(const double2* __restrict__ U, Lat g, const double2* __restrict__ x, double2* y, double2* t0,
                   double2* t1, int deg, double c, double a, GridBar* bar, int* herr) {
  extern __shared__ double2 s_ub[];  // [27][128] backward links (RESIDENT only)
  double2 (*sUb)[128] = reinterpret_cast<double2 (*)[128]>(s_ub);
  const unsigned nblk = gridDim.x;
  // T_n lives in buffer (2 - (deg - n)) mod 3 of {t0, t1, y}: T_deg lands in y
  auto buf = [=](int n) {
    const int i = (((2 - (deg - n)) % 3) + 3) % 3;
    return i == 0 ? t0 : (i == 1 ? t1 : y);
  };
  const double cd = a - 6.0 * c;
  int s = blockIdx.x * 128 + threadIdx.x;
  double2 uf[3][9];
  int up[3], dn[3];
  if (RESIDENT) {
    if (s < g.V3) {
      int sx, sy, sz;
      site_xyz(g, s, sx, sy, sz);
#pragma unroll
      for (int mu = 0; mu < 3; ++mu) {
        up[mu] = nb_up(g, sx, sy, sz, mu);
        dn[mu] = nb_dn(g, sx, sy, sz, mu);
#pragma unroll
        for (int e = 0; e < 9; ++e) {
          uf[mu][e] = __ldg(U + (size_t)(mu * 9 + e) * g.V3 + s);
          sUb[mu * 9 + e][threadIdx.x] = __ldg(U + (size_t)(mu * 9 + e) * g.V3 + dn[mu]);
        }
      }
    }
  }
  for (int n = 1; n <= deg; ++n) {
    const double2* X = n == 1 ? x : buf(n - 1);
    const double2* Z = n == 2 ? x : (n > 2 ? buf(n - 2) : nullptr);
    double2* Y = buf(n);
    const double ch = n == 1 ? c : 2.0 * c, cdiag = n == 1 ? cd : 2.0 * cd;
    for (int si = s; si < g.V3; si += (RESIDENT ? g.V3 : (int)nblk * 128)) {
      if (!RESIDENT) {
        int sx, sy, sz;
        site_xyz(g, si, sx, sy, sz);
#pragma unroll
        for (int mu = 0; mu < 3; ++mu) {
          up[mu] = nb_up(g, sx, sy, sz, mu);
          dn[mu] = nb_dn(g, sx, sy, sz, mu);
        }
      }
      double2 acc[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
#pragma unroll
      for (int mu = 0; mu < 3; ++mu) {
        double2 xu[3], xd[3];
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          xu[b] = n == 1 ? __ldg(X + 3 * (size_t)up[mu] + b) : __ldcg(X + 3 * (size_t)up[mu] + b);
          xd[b] = n == 1 ? __ldg(X + 3 * (size_t)dn[mu] + b) : __ldcg(X + 3 * (size_t)dn[mu] + b);
        }
#pragma unroll
        for (int aa = 0; aa < 3; ++aa)
#pragma unroll
          for (int b = 0; b < 3; ++b) {
            if (RESIDENT) {
              cfma(acc[aa], uf[mu][3 * aa + b], xu[b]);
              cfmac(acc[aa], sUb[mu * 9 + 3 * b + aa][threadIdx.x], xd[b]);
            } else {
              cfma(acc[aa], __ldg(U + (size_t)(mu * 9 + 3 * aa + b) * g.V3 + si), xu[b]);
              cfmac(acc[aa], __ldg(U + (size_t)(mu * 9 + 3 * b + aa) * g.V3 + dn[mu]), xd[b]);
            }
          }
      }
#pragma unroll
      for (int aa = 0; aa < 3; ++aa) {
        const double2 xs = n == 1 ? __ldg(X + 3 * (size_t)si + aa) : __ldcg(X + 3 * (size_t)si + aa);
        double2 r = make_double2(ch * acc[aa].x + cdiag * xs.x, ch * acc[aa].y + cdiag * xs.y);
        if (Z) {
          const double2 zz = n == 2 ? __ldg(Z + 3 * (size_t)si + aa) : __ldcg(Z + 3 * (size_t)si + aa);
          r.x -= zz.x;
          r.y -= zz.y;
        }
        __stcg(Y + 3 * (size_t)si + aa, r);
      }
    }
    if (n < deg && !grid_barrier(bar, nblk, herr)) return;
  }
}

namespace {
struct FusedOcc {
  int sms = 0, res = 0, nonres = 0;
};
std::mutex g_fused_mu;
FusedOcc g_fused_occ[64];

int fused_occupancy(FusedOcc* out) {
  int dev = 0;
  LAPH_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    set_error("device ordinal %d not supported", dev);
    return LAPH_EINVAL;
  }
  std::lock_guard<std::mutex> lk(g_fused_mu);
  FusedOcc& o = g_fused_occ[dev];
  if (o.sms == 0) {
    LAPH_CUDA_TRY(cudaFuncSetAttribute(k_cheb64_fused<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kFusedSmem));
    LAPH_CUDA_TRY(cudaDeviceGetAttribute(&o.sms, cudaDevAttrMultiProcessorCount, dev));
    LAPH_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o.res, k_cheb64_fused<true>, 128, kFusedSmem));
    LAPH_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o.nonres, k_cheb64_fused<false>, 128, 0));
  }
  *out = o;
  return LAPH_OK;
}
}  // namespace

int cheb64_fused(const double2* U, int L, double lam_l, double lam_c, int deg, const double2* x, double2* y,
                 double2* tmp, size_t ld, GridBar* bar, int* herr, cudaStream_t st) {
  const double c = 2.0 / (lam_l - lam_c);
  const double a = 1.0 + c * lam_c;
  const Lat g = make_lat(L);
  if (deg <= 1) return hop64(U, L, x, nullptr, y, ld, 1, c, a - 6.0 * c, 0.0, st);
  FusedOcc o;
  LAPH_TRY(fused_occupancy(&o));
  const int need = (int)ceil_div(g.V3, 128);
  const bool resident = need <= o.res * o.sms;
  const int grid = resident ? need : std::max(1, std::min(need, o.nonres * o.sms));
  if (grid < 1 || (!resident && o.nonres < 1)) {
    set_error("cheb64_fused: no co-resident grid for L = %d", L);
    return LAPH_ECUDA;
  }
  // the barrier's counter is left ready by every completed launch (its owner
  // resets it only after a barrier gave up)
  double2* t0 = tmp;
  double2* t1 = tmp + ld;
  Lat gg = g;
  void* args[] = {(void*)&U, (void*)&gg, (void*)&x, (void*)&y, (void*)&t0, (void*)&t1, (void*)&deg, (void*)&c,
                  (void*)&a, (void*)&bar, (void*)&herr};
  if (resident)
    LAPH_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)k_cheb64_fused<true>, dim3(grid), dim3(128), args,
                                              kFusedSmem, st));
  else
    LAPH_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)k_cheb64_fused<false>, dim3(grid), dim3(128), args, 0, st));
  return LAPH_OK;
}

}  // namespace laph

// The architecture the library's device code was built for, as the CUDA
// runtime reports it for one of its kernels (cudaFuncAttributes::binaryVersion,
// major * 10 + minor: 100 for sm_100a).
extern "C" int laph_binary_version(int* version) {
  if (!version) {
    laph::set_error("laph_binary_version: null pointer");
    return LAPH_EINVAL;
  }
  cudaFuncAttributes fa;
  const cudaError_t e = cudaFuncGetAttributes(&fa, laph::k_hop64<false>);
  if (e != cudaSuccess) {
    cudaGetLastError();
    laph::set_error("laph_binary_version: %s", cudaGetErrorString(e));
    return e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? LAPH_ENODEV : LAPH_ECUDA;
  }
  *version = fa.binaryVersion;
  return LAPH_OK;
}
