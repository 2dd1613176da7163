// sourceshape.cu -- the distillation source shape psi(r) of one timeslice's
// eigenvectors on the device (the reference's sourceshape program:
// modules/sourceshape_funcs.cpp:30-81, src/sourceshape.cpp):
//
//   psi(r) = sum_x || V_{x+r} V_x^dag ||_F ,  r_i = 0, 2, ..., L-2,
//
// V_y the 3 x nev block of the eigensystem's rows 3y .. 3y+2.  Since every r
// is even, x and x+r share their coordinate parities, so the 3x3 blocks needed
// are exactly the diagonal blocks P_cc = V_c V_c^dag of the projector V V^dag
// restricted to each of the 8 parity classes c of sites.  Each class is a
// complex GEMM of (3 V3/8) x (3 V3/8) over K = nev; P_cc is Hermitian and
// ||P_xy||_F = ||P_yx||_F, so only upper tile pairs are formed and an
// off-diagonal tile adds each norm to the bins of r and -r.  The epilogue
// turns every 3x3 block into its Frobenius norm and bins it by r = y - x.
//
//   k_ss_pack : V (column-major [3 V3][nev]) -> class-major Vp[c][n][3 s_c + colour]
//               (optionally columns weighted by sqrt|ev|, weight_eigenvectors
//               of sourceshape_funcs.cpp:85-96)
//   k_ss_tile : one CTA per (class, upper 32x32 site-tile pair): FP64 tile
//               GEMM through a 2-stage cp.async ring, norms, per-CTA shared
//               bins (L <= 32) flushed with one atomic per touched bin.  The
//               product runs on the FP64 tensor path (mma m8n8k4, 16 warps of
//               24 x 24 rows x columns, four real MMAs per complex one) by
//               default; LAPH_SOURCESHAPE_KERNEL=0 selects the FP64-FMA form
//               (one thread per 2 x 1 site pairs, 18 complex accumulators).
//
// FP64 throughout (parity with the FP64 reference to 1e-12 relative); the
// bins are summed with atomics, so the last bits depend on the order.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "batch.cuh"
#include "common.cuh"

namespace laph {
namespace {

// d(8x8, 2 per thread) += a(8x4, 1 per thread) b(4x8, 1 per thread), FP64 tensor MMA
// (not volatile: the compiler may schedule it; issued accumulator-major below)
__device__ __forceinline__ void dmma884(double (&acc)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(acc[0]), "+d"(acc[1])
      : "d"(a), "d"(b));
}

constexpr int kSsSites = 32;               // sites per tile side
constexpr int kSsRows = 3 * kSsSites;      // rows per tile side
constexpr int kSsK = 8;                    // eigenvectors per pipeline stage
constexpr int kSsStage = 2 * kSsK * kSsRows;  // double2 per stage (A and B)
constexpr int kSsBinsMax = 4096;           // shared bins: (L/2)^3 <= 4096, i.e. L <= 32
constexpr int kSsSmem = 2 * kSsStage * (int)sizeof(double2) + kSsBinsMax * (int)sizeof(double);

__global__ void k_ss_pack(const double2* __restrict__ V, int L, int nev, const double* __restrict__ evals,
                          double2* __restrict__ Vp, int cm) {
  const int H = L / 2, Nc = H * H * H, R = 3 * Nc;
  const long long dim = 3LL * L * L * L;
  const long long total = 8LL * nev * R;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % R);
    const long long cn = e / R;
    const int n = (int)(cn % nev), c = (int)(cn / nev);
    const int sc = i / 3, colour = i - 3 * sc;
    const int a = sc / (H * H), b = (sc / H) % H, cc = sc % H;
    const int x = 2 * a + (c >> 2), y = 2 * b + ((c >> 1) & 1), z = 2 * cc + (c & 1);
    const long long site = (long long)x * L * L + y * L + z;
    // input 3*site + colour, or colour-major (cm: colour*V3 + site, the solver's own blocks)
    double2 v = V[(cm ? colour * (dim / 3) + site : 3 * site + colour) + n * dim];
    if (evals) {
      const double w = sqrt(fabs(evals[n]));
      v = make_double2(v.x * w, v.y * w);
    }
    Vp[e] = v;
  }
}

// kDmma: the tile product on the FP64 tensor path (mma m8n8k4), else FP64 FMAs with one
// thread per site pair
template <bool kDmma>
__global__ void __launch_bounds__(512, 1) k_ss_tile(const double2* __restrict__ Vp, int L, int nev,
                                                 double* __restrict__ psi) {
  const int H = L / 2, Nc = H * H * H, R = 3 * Nc;
  const int T = (Nc + kSsSites - 1) / kSsSites;
  const int npair = T * (T + 1) / 2;
  const int c = blockIdx.x / npair;
  int pr = blockIdx.x - c * npair, ty = 0;
  while (pr >= T - ty) {
    pr -= T - ty;
    ++ty;
  }
  const int tx = ty + pr;
  const double2* Vc = Vp + (size_t)c * nev * R;
  extern __shared__ double2 ssm[];
  double* bins = reinterpret_cast<double*>(ssm + 2 * kSsStage);
  const int nbins = H * H * H;
  const bool shared_bins = nbins <= kSsBinsMax;
  if (shared_bins)
    for (int b = threadIdx.x; b < nbins; b += blockDim.x) bins[b] = 0.0;
  // stage layout: A[kSsK][kSsRows] (rows of tile ty), B[kSsK][kSsRows] (rows of tile tx)
  const int rowA = ty * kSsRows, rowB = tx * kSsRows;
  auto load = [&](int n0, int st) {
    double2* A = ssm + st * kSsStage;
    double2* B = A + kSsK * kSsRows;
    for (int e = threadIdx.x; e < kSsK * kSsRows; e += blockDim.x) {
      const int q = e / kSsRows, j = e - q * kSsRows;
      const int n = n0 + q;
      const bool okA = n < nev && rowA + j < R, okB = n < nev && rowB + j < R;
      cp_async16(A + e, Vc + (okA ? (size_t)n * R + rowA + j : 0), okA);
      cp_async16(B + e, Vc + (okB ? (size_t)n * R + rowB + j : 0), okB);
    }
    cp_async_commit();
  };
  if constexpr (kDmma) {
  // FP64 tensor path: the tile pair is a 96 x 96 complex product P = A B^H over
  // K = nev; warp (wr, wc) of the 4 x 4 warp grid owns the 24 x 24 block of
  // rows 24 wr.., columns 24 wc.. (8 x 8 site pairs, 3 x 3 MMA tiles of 8 x 8);
  // a conj(b) = (ar br + ai bi) + i (ai br - ar bi) as four real MMAs.
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wr = warp >> 2, wc = warp & 3;
  const int fr = lane >> 2, fk = lane & 3;
  double accr[3][3][2], acci[3][3][2];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) accr[i][j][0] = accr[i][j][1] = acci[i][j][0] = acci[i][j][1] = 0.0;
  const int nstep = (nev + kSsK - 1) / kSsK;
  load(0, 0);
  for (int it = 0; it < nstep; ++it) {
    const int st = it & 1;
    if (it + 1 < nstep) {
      load((it + 1) * kSsK, st ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const double2* A = ssm + st * kSsStage;
    const double2* B = A + kSsK * kSsRows;
#pragma unroll
    for (int ks = 0; ks < kSsK / 4; ++ks) {
      const int q = 4 * ks + fk;
      double ar[3], ai[3], br[3], bi[3], bn[3];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const double2 a = A[q * kSsRows + 24 * wr + 8 * i + fr];
        ar[i] = a.x;
        ai[i] = a.y;
      }
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const double2 b = B[q * kSsRows + 24 * wc + 8 * j + fr];
        br[j] = b.x;
        bi[j] = b.y;
        bn[j] = -b.y;
      }
      // accumulator-major: consecutive MMAs never feed the same accumulator
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) dmma884(accr[i][j], ar[i], br[j]);
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) dmma884(acci[i][j], ai[i], br[j]);
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) dmma884(accr[i][j], ai[i], bi[j]);
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) dmma884(acci[i][j], ar[i], bn[j]);
    }
    __syncthreads();
  }
  // |P_ab|^2 summed per site pair in shared memory (the staging ring is free now)
  double* sq = reinterpret_cast<double*>(ssm) + warp * 64;  // [8 y sites][8 x sites] of this warp
  for (int e = lane; e < 64; e += 32) sq[e] = 0.0;
  __syncwarp();
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int rr = 8 * i + fr, cc = 8 * j + 2 * fk + e;  // within the warp's 24 x 24 block
        atomicAdd(&sq[(rr / 3) * 8 + cc / 3], accr[i][j][e] * accr[i][j][e] + acci[i][j][e] * acci[i][j][e]);
      }
  __syncwarp();
  for (int e = lane; e < 64; e += 32) {
    const int ys = ty * kSsSites + 8 * wr + e / 8, xs = tx * kSsSites + 8 * wc + e % 8;
    if (ys >= Nc || xs >= Nc) continue;
    const double f = sqrt(sq[e]);
    const int ay = ys / (H * H), by = (ys / H) % H, cy = ys % H;
    const int ax = xs / (H * H), bx = (xs / H) % H, cx = xs % H;
    const int da = ay - ax, db = by - bx, dc = cy - cx;
    const int r_fw = ((da + H) % H) * H * H + ((db + H) % H) * H + (dc + H) % H;
    if (shared_bins) atomicAdd(&bins[r_fw], f);
    else atomicAdd(&psi[r_fw], f);
    if (tx != ty) {
      const int r_bw = ((H - da) % H) * H * H + ((H - db) % H) * H + (H - dc) % H;
      if (shared_bins) atomicAdd(&bins[r_bw], f);
      else atomicAdd(&psi[r_bw], f);
    }
  }
  } else {
  // thread: y sites py, py + 16 of tile ty; x site px of tile tx (a warp shares py)
  const int py = threadIdx.x >> 5, px = threadIdx.x & 31;
  double2 acc[2][9];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int e = 0; e < 9; ++e) acc[i][e] = make_double2(0.0, 0.0);
  const int nstep = (nev + kSsK - 1) / kSsK;
  load(0, 0);
  for (int it = 0; it < nstep; ++it) {
    const int st = it & 1;
    if (it + 1 < nstep) {
      load((it + 1) * kSsK, st ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const double2* A = ssm + st * kSsStage;
    const double2* B = A + kSsK * kSsRows;
#pragma unroll
    for (int q = 0; q < kSsK; ++q) {
      double2 ya[2][3], xb[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        ya[0][a] = A[q * kSsRows + 3 * py + a];
        ya[1][a] = A[q * kSsRows + 3 * (py + 16) + a];
        xb[a] = B[q * kSsRows + 3 * px + a];
      }
      // M_ab += V_y[a] conj(V_x[b])
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int b = 0; b < 3; ++b) cfmac(acc[i][3 * a + b], xb[b], ya[i][a]);
    }
    __syncthreads();
  }
  // norms, binned by r = y - x (and x - y for off-diagonal tile pairs)
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int ys = ty * kSsSites + py + 16 * i, xs = tx * kSsSites + px;
    if (ys >= Nc || xs >= Nc) continue;
    double f = 0.0;
#pragma unroll
    for (int e = 0; e < 9; ++e) f += acc[i][e].x * acc[i][e].x + acc[i][e].y * acc[i][e].y;
    f = sqrt(f);
    const int ay = ys / (H * H), by = (ys / H) % H, cy = ys % H;
    const int ax = xs / (H * H), bx = (xs / H) % H, cx = xs % H;
    const int da = ay - ax, db = by - bx, dc = cy - cx;
    const int r_fw = ((da + H) % H) * H * H + ((db + H) % H) * H + (dc + H) % H;
    if (shared_bins) atomicAdd(&bins[r_fw], f);
    else atomicAdd(&psi[r_fw], f);
    if (tx != ty) {
      const int r_bw = ((H - da) % H) * H * H + ((H - db) % H) * H + (H - dc) % H;
      if (shared_bins) atomicAdd(&bins[r_bw], f);
      else atomicAdd(&psi[r_bw], f);
    }
  }
  }
  if (shared_bins) {
    __syncthreads();
    for (int b = threadIdx.x; b < nbins; b += blockDim.x)
      if (bins[b] != 0.0) atomicAdd(&psi[b], bins[b]);
  }
}

bool g_ss_attr[64] = {false};

// LAPH_SOURCESHAPE_KERNEL=0 selects the FP64-FMA tile kernel, 1 (default) the FP64 tensor-path one
bool ss_use_dmma() {
  static const bool v = [] {
    const char* e = std::getenv("LAPH_SOURCESHAPE_KERNEL");
    return !(e && e[0] == '0');
  }();
  return v;
}

}  // namespace

// psi[(L/2)^3] (device) from a device eigensystem V [3 V3][nev] (column stride 3 V3,
// colour-major rows when cm); work: 8 nev (3 V3 / 8) double2 of device scratch owned by the caller.
int sourceshape_device(const double2* V, int L, int nev, const double* evals, double2* work, double* psi, int cm,
                       cudaStream_t st) {
  int dev = 0;
  LAPH_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 64 && !g_ss_attr[dev]) {
    LAPH_CUDA_TRY(cudaFuncSetAttribute(k_ss_tile<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSsSmem));
    LAPH_CUDA_TRY(cudaFuncSetAttribute(k_ss_tile<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSsSmem));
    g_ss_attr[dev] = true;
  }
  const int H = L / 2, Nc = H * H * H;
  const int T = (Nc + kSsSites - 1) / kSsSites;
  LAPH_CUDA_TRY(cudaMemsetAsync(psi, 0, sizeof(double) * Nc, st));
  const long long total = 8LL * nev * 3 * Nc;
  const int pb = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
  k_ss_pack<<<pb, 256, 0, st>>>(V, L, nev, evals, work, cm);
  LAPH_CUDA_TRY(cudaGetLastError());
  if (ss_use_dmma())
    k_ss_tile<true><<<8 * T * (T + 1) / 2, 512, kSsSmem, st>>>(work, L, nev, psi);
  else
    k_ss_tile<false><<<8 * T * (T + 1) / 2, 512, kSsSmem, st>>>(work, L, nev, psi);
  LAPH_CUDA_TRY(cudaGetLastError());
  return LAPH_OK;
}

}  // namespace laph

using namespace laph;

extern "C" int laph_sourceshape(const double* V, int L, int nev, const double* evals, int on_device, double* psi,
                                int device) {
  if (!V || !psi || L < 2 || (L & 1) || nev < 1) {
    set_error("laph_sourceshape: bad argument (need V, psi, an even L >= 2 and nev >= 1)");
    return LAPH_EINVAL;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    set_error("laph_sourceshape: no CUDA device %d", device);
    return LAPH_ENODEV;
  }
  LAPH_CUDA_TRY(cudaSetDevice(device));
  const long long dim = 3LL * L * L * L;
  const int H = L / 2, Nc = H * H * H;
  double2 *dV = nullptr, *work = nullptr;
  double *dpsi = nullptr, *dev_ev = nullptr;
  cudaStream_t st = nullptr;
  int rc = LAPH_OK;
  auto cleanup = [&]() {
    if (st) cudaStreamSynchronize(st);
    if (!on_device) {
      cudaFree(dV);
      cudaFree(dev_ev);
    }
    cudaFree(work);
    cudaFree(dpsi);
    if (st) cudaStreamDestroy(st);
  };
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&work, sizeof(double2) * dim * nev) != cudaSuccess ||
      cudaMalloc(&dpsi, sizeof(double) * Nc) != cudaSuccess) {
    cudaGetLastError();
    cleanup();
    set_error("laph_sourceshape: device allocation failed");
    return LAPH_ENOMEM;
  }
  const double2* Vuse = reinterpret_cast<const double2*>(V);
  const double* ev_use = evals;
  if (!on_device) {
    if (cudaMalloc(&dV, sizeof(double2) * dim * nev) != cudaSuccess ||
        (evals && cudaMalloc(&dev_ev, sizeof(double) * nev) != cudaSuccess)) {
      cudaGetLastError();
      cleanup();
      set_error("laph_sourceshape: device allocation failed");
      return LAPH_ENOMEM;
    }
    if (cudaMemcpyAsync(dV, V, sizeof(double2) * dim * nev, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        (evals && cudaMemcpyAsync(dev_ev, evals, sizeof(double) * nev, cudaMemcpyHostToDevice, st) != cudaSuccess)) {
      cudaGetLastError();
      cleanup();
      set_error("laph_sourceshape: host to device copy failed");
      return LAPH_ECUDA;
    }
    Vuse = dV;
    ev_use = dev_ev;
  }
  rc = sourceshape_device(Vuse, L, nev, ev_use, work, dpsi, 0, st);
  if (rc == LAPH_OK && (cudaMemcpyAsync(psi, dpsi, sizeof(double) * Nc, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                        cudaStreamSynchronize(st) != cudaSuccess)) {
    set_error("laph_sourceshape: %s", cudaGetErrorString(cudaGetLastError()));
    rc = LAPH_ECUDA;
  }
  cleanup();
  return rc;
}
