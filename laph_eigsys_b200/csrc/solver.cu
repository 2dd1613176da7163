// solver.cu -- the batched block eigensolver (laph_solver_*): a device-resident
// Chebyshev-filtered subspace iteration over many timeslices at once.
//
// Per problem (timeslice), with A = -Delta, block width k = nev + guard
// (rounded up to a multiple of 32), FP64 Ritz block V, Ritz values Theta and
// FP64 residuals R = A V - V Theta:
//   1. filter   W = T_m(B) V with B = c_hop hop + c_diag mapping the damped
//               interval [lam_cut, lam_max] to [-1, 1].  The exact part
//               V T_m(Theta_B) is formed in FP64; only the correction E_m,
//               driven by S = 2(B V - V Theta_B) = -2 c_hop R, runs through
//               the FP32 multi-RHS stencil (lap_cheb_mrhs), so FP32 rounding
//               scales with |R| and the iteration converges to FP64 accuracy.
//   2. Y = A W  (FP64 stencil)
//   3. [G | H] = W^H [W | Y]  (FP64)
//   4. per problem: scaled Cholesky G = D R^H R D, Minv = D^-1 R^-1,
//      Jacobi eigensolve of Minv^H H Minv = Q Theta Q^H, C = Minv Q,
//      next window lam_cut = max Ritz value, Chebyshev coefficient table
//   5. V = W C, R = Y C - V Theta, S = -2 c_hop R (FP32), residual norms
//   6. convergence mask: all nev wanted ||r_j|| / lam_max <= tol
// Every step is one launch over all active problems (CTA -> problem through a
// prefix table), so the host loop issues the same launches each iteration.
// This replaces, per timeslice, MatCreateShell + EPSSolve + EPSGetEigenpair +
// fix_phase + recover_spectrum of the reference (src/ev_ts.cpp:197-319).
#include <algorithm>
#include <cmath>
#include <map>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "batch.cuh"
#include "common.cuh"
#include "dense.cuh"
#include "filter.cuh"
#include "links.cuh"
#include "loop.cuh"
#include "mlp.cuh"
#include "smear.cuh"
#include "stencil64cols.cuh"

namespace laph {
int displace_device(const double2* U, int L, int dir, int nev, long long ldv, const double2* V, double2* W, int cm,
                    cudaStream_t st);
int sourceshape_device(const double2* V, int L, int nev, const double* evals, double2* work, double* psi, int cm,
                       cudaStream_t st);
}

using namespace laph;

struct laph_solver {
  int dev = 0;
  cudaStream_t st = nullptr;
  laph_solve_opts o{};
  int np = 0, mdeg = 16, kb = 32, tile = 128;
  int fvariant = 1, lmax = 0;  // filter variant in use (opts.filter_kernel, or 1 where 3 does not apply)
  int* d_ferr = nullptr;       // set by the staged filter when a pipeline wait gives up
  std::vector<ProbDesc> hd;
  ProbDesc* d_pd = nullptr;
  ProbState* d_ps = nullptr;
  std::vector<ProbState> hps;
  // CTA -> problem prefix tables
  int *st_site = nullptr, *st_filt = nullptr, *st_nl = nullptr, *st_res = nullptr, *st_gram = nullptr, *st_gred = nullptr,
      *st_rot = nullptr, *st_rand = nullptr, *st_col = nullptr;
  int nb_site = 0, nb_filt = 0, nb_nl = 0, nb_res = 0, nb_gram = 0, nb_gred = 0, nb_rot = 0, nb_rand = 0, nb_col = 0;
  // pools
  double2 *U64raw = nullptr, *U64 = nullptr, *Utmp = nullptr, *dec = nullptr, *stage = nullptr;
  float2* Uf32 = nullptr;
  void* Ubf = nullptr;
  float* scale = nullptr;
  double2 *V = nullptr, *W = nullptr, *Y = nullptr;
  float2 *S = nullptr, *E[3] = {nullptr, nullptr, nullptr};
  double2 *KK = nullptr, *gpart = nullptr;
  double *rpart = nullptr, *theta = nullptr, *tcoef = nullptr, *scol = nullptr, *dwork = nullptr, *resid = nullptr,
         *phases = nullptr, *norms = nullptr;
  int* d_nactive = nullptr;
  int* h_nactive = nullptr;
  unsigned long long* tstamp = nullptr;  // [np][kSmallPhases] phase boundaries of the small dense step
  size_t blk_total = 0;
  std::vector<int> links_set;
  std::vector<double> sp1, sp2;  // per-problem smearing parameters (opts' by default)
  std::vector<int> degs;  // filter degree of each pass of the last run
  std::vector<double> lam_max0;  // top of the first pass's window, per problem
  std::vector<int> fallback;     // learned first window failed its check, per problem
  double ms[4] = {0, 0, 0, 0};
  long long cnt[3] = {0, 0, 0};
  // algorithmic bytes of the filter passes of the last run: [0] what the
  // kernels must move (X, Z, S read, Y written, FP64 V / W in the last step,
  // W = V for locked columns, links once per column block), [1] the unit
  // 72 B + links / block per unlocked site-vector-step (X, Z read, Y written)
  double fbytes[2] = {0, 0};
  std::vector<cudaEvent_t> evf;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
  int ran = 0;
  // learned window / features
  float* model = nullptr;   // device: params + normalisation
  int have_model = 0;
  float *feats = nullptr, *mwork = nullptr;
  double *bound = nullptr, *plaq = nullptr;
  int* wdeg = nullptr;
  int deg0 = 0;             // degree cap of the first filter pass from the model
  // CUDA graphs of one outer iteration: the filter pass (one per degree) and
  // the Rayleigh-Ritz pass, captured on first use and replayed
  std::map<int, cudaGraphExec_t> g_filter;
  cudaGraphExec_t g_rr = nullptr;
  // device-side loop: the whole solve as one graph (setup, a WHILE node over
  // the outer iteration with a SWITCH node per filter step, phase fix)
  LoopState* ls = nullptr;
  int* d_degs = nullptr;                           // degree of each pass
  double* d_lam_max0 = nullptr;                    // first pass's lam_max per problem
  int* d_fallback = nullptr;                       // learned window fell back, per problem
  cudaGraphConditionalHandle* d_steps = nullptr;   // [mdeg] SWITCH handles of the filter steps
  ProbState* d_ps0 = nullptr;                      // state every run starts from
  cudaGraphExec_t g_solve = nullptr;
  long long solve_setup_launches = 0;              // kernels of the graph outside the loop
  int solve_graph_failed = 0;                      // capture refused: the host loop from then on
  int last_loop = 0;                               // the last run: 1 device-side loop (one launch), 0 host loop
  long long last_graph_launches = 0;               // graph launches the last run made
  // asynchronous read-back (laph_solver_get_async): a conversion stream (out
  // of V into a device staging pool the runs never touch) and a copy stream
  // (staging pool -> host), so the copies of one run's results overlap the
  // next run, which waits only for the conversions
  cudaStream_t st_conv = nullptr, st_out = nullptr;
  std::vector<cudaEvent_t> ev_ready, ev_copied;  // per problem: converted / copied out
  std::vector<int> copied_rec;                    // ev_copied[i] has been recorded
  double2* out_vec = nullptr;   // reference-layout eigenvectors, sum of dim x nev
  double* out_val = nullptr;    // eigenvalues (recover_spectrum sign) and phases, 2 x sum of nev
  std::vector<size_t> out_off;  // per problem: offset of its block in out_vec
  std::vector<size_t> out_voff; // per problem: offset of its 2 nev values in out_val
  cudaEvent_t ev_run = nullptr, ev_conv = nullptr;
  int conv_pending = 0;
};

namespace {

template <typename T>
int dalloc(T** p, size_t n) {
  if (n == 0) n = 1;
  if (cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    set_error("device allocation of %zu bytes failed", n * sizeof(T));
    return LAPH_ENOMEM;
  }
  return LAPH_OK;
}

int upload_prefix(const std::vector<int>& per, int** d, int* total) {
  std::vector<int> pre(per.size() + 1, 0);
  for (size_t i = 0; i < per.size(); ++i) pre[i + 1] = pre[i] + per[i];
  *total = pre.back();
  LAPH_TRY(dalloc(d, pre.size()));
  LAPH_CUDA_TRY(cudaMemcpy(*d, pre.data(), pre.size() * sizeof(int), cudaMemcpyHostToDevice));
  return LAPH_OK;
}

int round_up(int a, int b) { return (a + b - 1) / b * b; }

}  // namespace

extern "C" {

// default laph_solve_opts.direct_resid: passes whose largest wanted residual (relative to lam_max) is above
// it filter V directly in FP32; the FP32 rounding of T_m(B)V (about m * 6e-8 relative) stays far below it.
// 1e-4 also takes the pass that brings the first columns to the locking threshold and delays locking:
// measured slower than 1e-3 (26.8 against 27.6 timeslices/s at 32^3 x 64, same box)
constexpr double kDirectResid = 1e-3;
// The threshold a solve uses: none with BF16 links, whose rounding (about 4e-3 relative) would put the
// direct filter's operator itself that far from B.
static double direct_resid(const laph_solve_opts& o) {
  return o.link_prec == LAPH_LINKS_BF16 ? -1.0 : o.direct_resid;
}

void laph_solve_opts_default(laph_solve_opts* o) {
  std::memset(o, 0, sizeof *o);
  o->smear_kind = LAPH_SMEAR_NONE;
  o->guard = 16;
  o->link_prec = LAPH_LINKS_FP32;
  o->tol = 1e-9;
  o->max_it = 200;
  o->window = LAPH_WINDOW_LANCZOS;
  o->deg = 16;
  o->phase_fix = 1;
  o->seed = 1227;
  o->filter_kernel = 1;
  o->direct_resid = kDirectResid;
}

int laph_solver_destroy(laph_solver* s) {
  if (!s) return LAPH_OK;
  cudaSetDevice(s->dev);
  if (s->st) cudaStreamSynchronize(s->st);
  void* ptrs[] = {s->d_pd, s->d_ps, s->st_site, s->st_filt, s->st_nl, s->st_res, s->st_gram, s->st_gred, s->st_rot, s->st_rand,
                  s->st_col, s->U64raw, s->U64, s->Utmp, s->dec, s->stage, s->Uf32, s->Ubf, s->scale, s->V, s->W, s->Y, s->S, s->E[0],
                  s->E[1], s->E[2], s->KK, s->gpart, s->rpart, s->theta, s->tcoef, s->scol, s->dwork, s->resid,
                  s->phases, s->norms, s->d_nactive, s->model, s->feats, s->mwork, s->bound, s->plaq, s->wdeg,
                  s->tstamp, s->ls, s->d_degs, s->d_lam_max0, s->d_fallback, s->d_steps, s->d_ps0, s->d_ferr};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (s->h_nactive) cudaFreeHost(s->h_nactive);
  if (s->st_out) cudaStreamSynchronize(s->st_out);
  if (s->st_conv) cudaStreamSynchronize(s->st_conv);
  for (auto e : s->ev_ready) cudaEventDestroy(e);
  for (auto e : s->ev_copied) cudaEventDestroy(e);
  if (s->st_conv) cudaStreamDestroy(s->st_conv);
  if (s->out_vec) cudaFree(s->out_vec);
  if (s->out_val) cudaFree(s->out_val);
  if (s->ev_run) cudaEventDestroy(s->ev_run);
  if (s->ev_conv) cudaEventDestroy(s->ev_conv);
  if (s->st_out) cudaStreamDestroy(s->st_out);
  for (auto& kv : s->g_filter) cudaGraphExecDestroy(kv.second);
  if (s->g_rr) cudaGraphExecDestroy(s->g_rr);
  if (s->g_solve) cudaGraphExecDestroy(s->g_solve);
  for (auto e : s->evf) cudaEventDestroy(e);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  if (s->ev2) cudaEventDestroy(s->ev2);
  if (s->st) cudaStreamDestroy(s->st);
  delete s;
  return LAPH_OK;
}

int laph_solver_create(laph_solver** out, const laph_problem* probs, int n, const laph_solve_opts* opts, int device) {
  if (!out || !probs || n < 1 || !opts) {
    set_error("laph_solver_create: bad argument");
    return LAPH_EINVAL;
  }
  if (opts->deg < 2 || opts->deg > kMaxFilterDeg || opts->guard < 0 || !(opts->tol > 0.0) || opts->max_it < 1 ||
      opts->block < 0 || opts->block > 512 || opts->filter_kernel < 0 || opts->filter_kernel > 5 ||
      (opts->filter_tile != 0 && opts->filter_tile != 64 && opts->filter_tile != 128 && opts->filter_tile != 256) ||
      !std::isfinite(opts->direct_resid)) {
    set_error("laph_solver_create: need 2 <= deg <= 128, guard >= 0, tol > 0, max_it >= 1, 0 <= block <= 512, "
              "filter_kernel in {0, ..., 5}, filter_tile in {0, 64, 128, 256}, finite direct_resid");
    return LAPH_EINVAL;
  }
  for (int i = 0; i < n; ++i) {
    const int L = probs[i].L, nev = probs[i].nev;
    const int k = round_up(nev + opts->guard, kGramTile);
    if (L < 3 || L > 128 || nev < 1 || k > 512 || k > 3 * L * L * L / 2) {
      set_error("laph_solver_create: problem %d: need 3 <= L <= 128, 1 <= nev, block width %d <= min(512, dim/2)", i, k);
      return LAPH_EINVAL;
    }
  }
  // every argument is checked before the device, so a bad call reports LAPH_EINVAL on any host
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("laph_solver_create: no CUDA device");
    return LAPH_ENODEV;
  }
  laph_solver* s = new laph_solver();
  auto fail = [&](int stt) {
    laph_solver_destroy(s);
    return stt;
  };
  s->dev = device;
  s->o = *opts;
  s->np = n;
  s->mdeg = opts->deg;
  s->kb = opts->block > 0 ? opts->block : 32;
  // sites per CTA of the filter; the per-thread-coefficient variant and blocks wider than 64 keep 128
  s->tile = opts->filter_tile > 0 && opts->filter_kernel >= 1 && s->kb <= 64 ? opts->filter_tile : 128;
  // the staged variant (3) needs 128-site tiles of whole z-rows inside one plane for every problem
  s->fvariant = opts->filter_kernel;
  for (int i = 0; i < n; ++i) s->lmax = std::max(s->lmax, probs[i].L);
  if (s->fvariant >= 3) {  // staged rows (3) or 512-site bricks (4): L in {16, 32, 64, 128} for every problem
    bool ok = s->kb <= 64;
    for (int i = 0; i < n; ++i) ok = ok && cheb_staged_ok(probs[i].L);
    if (ok) s->tile = s->fvariant == 4 ? 512 : 128;
    else s->fvariant = 1;
  }
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    set_error("laph_solver_create: cannot use device %d", device);
    return fail(LAPH_ECUDA);
  }
  if (int e = dense_init()) return fail(e);
  if (int e = cheb_init()) return fail(e);
  // descriptors and pool offsets
  long long o_u64 = 0, o_uf = 0, o_sc = 0, o_blk = 0, o_kk = 0, o_kv = 0, o_gp = 0, o_rp = 0, o_tc = 0;
  size_t max_run = 0, max_v3 = 0;
  std::vector<int> per_site, per_filt, per_nl, per_res, per_gram, per_gred, per_rot, per_rand, per_col;
  for (int i = 0; i < n; ++i) {
    ProbDesc d{};
    d.L = probs[i].L;
    d.V3 = d.L * d.L * d.L;
    d.dim = 3 * d.V3;
    d.nev = probs[i].nev;
    d.k = round_up(d.nev + opts->guard, kGramTile);
    d.mdeg = s->mdeg;
    d.u64 = o_u64;
    d.uf = o_uf;
    d.sc = o_sc;
    d.blk = o_blk;
    d.kk = o_kk;
    d.kv = o_kv;
    d.gp = o_gp;
    d.rp = o_rp;
    d.tc = o_tc;
    const int chunk_rows = 8192;
    d.nchunk = (d.dim + chunk_rows - 1) / chunk_rows;
    d.nrt = (d.V3 + 127) / 128;  // site tiles of the residual kernel
    const int T = d.k / kGramTile, npair = T * (T + 1) / 2;
    o_u64 += 27LL * d.V3;
    o_uf += 27LL * d.V3;
    o_sc += d.V3;
    o_blk += (long long)d.dim * d.k;
    o_kk += 5LL * d.k * d.k;
    o_kv += d.k;
    o_gp += (long long)d.nchunk * 2 * npair * kGramTile * kGramTile;
    o_rp += (long long)d.nrt * d.k;
    o_tc += (long long)(s->mdeg + 1) * 3 * d.k;
    s->hd.push_back(d);
    max_v3 = std::max(max_v3, (size_t)d.V3);
    const int nst = (d.V3 + 127) / 128;
    per_site.push_back(nst);
    per_filt.push_back(((d.V3 + s->tile - 1) / s->tile) * ((d.k + s->kb - 1) / s->kb));
    per_nl.push_back(nst * ((d.k + kColsFP64 - 1) / kColsFP64));
    per_res.push_back(nst * d.k);
    per_gram.push_back(d.nchunk * npair);
    per_gred.push_back((2 * npair * kGramTile * kGramTile + 255) / 256);
    per_rot.push_back(((d.dim + kRotRows - 1) / kRotRows) * (d.k / 32));
    per_rand.push_back((int)(((long long)d.dim * d.k + 255) / 256));
    per_col.push_back(d.nev);
  }
  // longest run of equal L (smearing is batched per run)
  for (int i = 0; i < n;) {
    int j = i;
    while (j < n && s->hd[j].L == s->hd[i].L) ++j;
    max_run = std::max(max_run, (size_t)(j - i) * 27 * s->hd[i].V3);
    i = j;
  }
  s->blk_total = (size_t)o_blk;
  int rc = LAPH_OK;
  if ((rc = dalloc(&s->d_pd, n)) || (rc = dalloc(&s->d_ps, n)) || (rc = dalloc(&s->U64, o_u64)) || (rc = dalloc(&s->U64raw, o_u64)) ||
      (rc = dalloc(&s->Utmp, max_run)) || (rc = dalloc(&s->stage, 36 * max_v3)) || (rc = dalloc(&s->dec, max_run * 2)) ||
      (rc = dalloc(&s->scale, o_sc)) || (rc = dalloc(&s->V, o_blk)) || (rc = dalloc(&s->W, o_blk)) ||
      (rc = dalloc(&s->Y, o_blk)) || (rc = dalloc(&s->S, o_blk)) || (rc = dalloc(&s->E[0], o_blk)) ||
      (rc = dalloc(&s->E[1], o_blk)) || (rc = dalloc(&s->E[2], o_blk)) || (rc = dalloc(&s->KK, o_kk)) ||
      (rc = dalloc(&s->gpart, o_gp)) || (rc = dalloc(&s->rpart, o_rp)) || (rc = dalloc(&s->theta, o_kv)) ||
      (rc = dalloc(&s->tcoef, o_tc)) || (rc = dalloc(&s->scol, o_kv)) || (rc = dalloc(&s->dwork, 4 * o_kv)) ||
      (rc = dalloc(&s->resid, o_kv)) || (rc = dalloc(&s->phases, o_kv)) || (rc = dalloc(&s->norms, o_kv)) ||
      (rc = dalloc(&s->d_nactive, 1)) || (rc = dalloc(&s->model, kMlpParams + kMlpNorm)) ||
      (rc = dalloc(&s->feats, (size_t)n * kMlpIn)) || (rc = dalloc(&s->mwork, (size_t)n * (kMlpIn + kMlpOut))) ||
      (rc = dalloc(&s->bound, n)) || (rc = dalloc(&s->plaq, 4 * (size_t)n)) || (rc = dalloc(&s->wdeg, n)) ||
      (rc = dalloc(&s->tstamp, (size_t)n * kSmallPhases)) || (rc = dalloc(&s->ls, 1)) ||
      (rc = dalloc(&s->d_degs, (size_t)opts->max_it + 2)) || (rc = dalloc(&s->d_lam_max0, n)) ||
      (rc = dalloc(&s->d_fallback, n)) || (rc = dalloc(&s->d_steps, (size_t)s->mdeg + 1)) ||
      (rc = dalloc(&s->d_ps0, n)) || (rc = dalloc(&s->d_ferr, 1)))
    return fail(rc);
  if (cudaMemset(s->d_ferr, 0, sizeof(int)) != cudaSuccess) return fail(LAPH_ECUDA);
  if (opts->link_prec == LAPH_LINKS_BF16) {
    if ((rc = dalloc(reinterpret_cast<float2**>(&s->Ubf), (size_t)o_uf))) return fail(rc);  // 4 B per element
  } else {
    if ((rc = dalloc(&s->Uf32, o_uf))) return fail(rc);
  }
  if (cudaMallocHost(&s->h_nactive, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    return fail(LAPH_ENOMEM);
  }
  if ((rc = upload_prefix(per_site, &s->st_site, &s->nb_site)) || (rc = upload_prefix(per_filt, &s->st_filt, &s->nb_filt)) ||
      (rc = upload_prefix(per_nl, &s->st_nl, &s->nb_nl)) || (rc = upload_prefix(per_res, &s->st_res, &s->nb_res)) || (rc = upload_prefix(per_gram, &s->st_gram, &s->nb_gram)) ||
      (rc = upload_prefix(per_gred, &s->st_gred, &s->nb_gred)) || (rc = upload_prefix(per_rot, &s->st_rot, &s->nb_rot)) ||
      (rc = upload_prefix(per_rand, &s->st_rand, &s->nb_rand)) || (rc = upload_prefix(per_col, &s->st_col, &s->nb_col)))
    return fail(rc);
  if (cudaMemcpy(s->d_pd, s->hd.data(), n * sizeof(ProbDesc), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    return fail(LAPH_ECUDA);
  }
  cudaEventCreate(&s->ev0);
  cudaEventCreate(&s->ev1);
  cudaEventCreate(&s->ev2);
  {
    // the state every run starts from (the spectrum of -Delta lies in [0, 12])
    std::vector<ProbState> ps0(n, ProbState{});
    for (auto& p : ps0) {
      p.lam_max = opts->lam_max > 0.0 ? opts->lam_max : 12.0;
      p.lam_cut = opts->lam_cut > 0.0 ? opts->lam_cut : 0.0;
      p.active = 1;
    }
    if (cudaMemcpy(s->d_ps0, ps0.data(), n * sizeof(ProbState), cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaGetLastError();
      return fail(LAPH_ECUDA);
    }
  }
  s->links_set.assign(n, 0);
  s->sp1.assign(n, opts->smear_p1);
  s->sp2.assign(n, opts->smear_p2);
  s->hps.assign(n, ProbState{});
  *out = s;
  return LAPH_OK;
}

int laph_solver_set_links(laph_solver* s, int i, const double* links, int layout, int on_device) {
  if (!s || i < 0 || i >= s->np || !links) {
    set_error("laph_solver_set_links: bad argument");
    return LAPH_EINVAL;
  }
  LAPH_CUDA_TRY(cudaSetDevice(s->dev));
  const ProbDesc& d = s->hd[i];
  double2* dst = s->U64raw + d.u64;  // pristine copy; run() smears a working copy
  if (on_device) {
    if (layout != LAPH_LAYOUT_ROWMAJOR && layout != LAPH_LAYOUT_CONF) {
      set_error("laph_solver_set_links: device links must be ROWMAJOR or CONF");
      return LAPH_EINVAL;
    }
    // device-side reorder to site-minor order through a host-free path:
    // copy to the scratch and transpose with a small kernel
    LAPH_TRY(links_to_soa_device(links, layout, d.V3, dst, s->st));
  } else if (layout == LAPH_LAYOUT_ROWMAJOR || layout == LAPH_LAYOUT_CONF) {
    // raw copy into the staging area, reorder on the device; the finiteness
    // scan of the host links runs while the copy is in flight
    const size_t n = (layout == LAPH_LAYOUT_CONF ? 36 : 27) * (size_t)d.V3;
    LAPH_CUDA_TRY(cudaMemcpyAsync(s->stage, links, n * sizeof(double2), cudaMemcpyHostToDevice, s->st));
    if (int e = check_links_finite(links, layout, d.V3, "laph_solver_set_links")) {
      cudaStreamSynchronize(s->st);  // leave no copy in flight; the stored links are unchanged
      return e;
    }
    LAPH_TRY(links_to_soa_device(reinterpret_cast<const double*>(s->stage), layout, d.V3, dst, s->st));
  } else {
    LAPH_TRY(check_links_finite(links, layout, d.V3, "laph_solver_set_links"));
    std::vector<double2> soa(27 * (size_t)d.V3);
    LAPH_TRY(links_to_soa(links, layout, d.V3, soa.data()));
    LAPH_CUDA_TRY(cudaMemcpyAsync(dst, soa.data(), soa.size() * sizeof(double2), cudaMemcpyHostToDevice, s->st));
    LAPH_CUDA_TRY(cudaStreamSynchronize(s->st));
  }
  s->links_set[i] = 1;
  return LAPH_OK;
}

// Largest wanted residual above which the filter's amplification is capped.
// Raising it to 5e-2 .. 1 lets the second pass run at the full degree and saves
// one outer iteration at 32^3 x 64, but the extra filter steps cost more than
// the Rayleigh-Ritz they save (20.3 against 21.0 timeslices/s).
constexpr double kCapResid = 1e-2;

// Largest wanted residual after the learned window's first pass that counts
// as a working window (the random start block has residuals of order 1).
constexpr double kWindowCheck = 0.2;

// R = A V - V Theta, S = -2 c_hop R and the residual partials: the column-block
// kernel by default, the one-thread-per-(site, column) kernel with
// LAPH_RESID_KERNEL=0 (both leave the same per-tile partials).
static int residual(laph_solver* s) {
  static const int kind = [] {
    const char* e = std::getenv("LAPH_RESID_KERNEL");
    return e && *e == '0' ? 0 : 1;
  }();
  if (kind == 0)
    return residual64(s->d_pd, s->d_ps, s->st_res, s->np, s->nb_res, s->U64, s->V, s->theta, s->S, s->rpart, s->st);
  return residual64_cols(s->d_pd, s->d_ps, s->st_nl, s->np, s->nb_nl, s->U64, s->V, s->theta, s->S, s->rpart, s->st);
}

static int iteration_rr(laph_solver* s, int first_iter) {
  const bool fixed = s->o.window == LAPH_WINDOW_FIXED && s->o.lam_cut > 0.0;
  LAPH_TRY(neglap64_batch(s->d_pd, s->d_ps, s->st_nl, s->np, s->nb_nl, s->U64, s->W, s->Y, s->st));
  LAPH_TRY(gram(s->d_pd, s->d_ps, s->st_gram, s->np, s->nb_gram, 8192, s->W, s->Y, s->gpart, s->st));
  LAPH_TRY(gram_reduce(s->d_pd, s->d_ps, s->st_gred, s->np, s->nb_gred, s->gpart, s->KK, s->st));
  LAPH_TRY(small_dense(s->d_pd, s->d_ps, s->np, s->KK, s->theta, s->tcoef, s->scol, s->dwork, first_iter, fixed ? 1 : 0,
                       s->o.jacobi_sweeps > 0 ? s->o.jacobi_sweeps : 2, s->tstamp, s->st));
  LAPH_TRY(rotate(s->d_pd, s->d_ps, s->st_rot, s->np, s->nb_rot, s->W, s->KK, s->V, s->st));
  LAPH_TRY(residual(s));
  LAPH_TRY(zero_int(s->d_nactive, s->st));
  LAPH_TRY(resid_check(s->d_pd, s->d_ps, s->np, s->rpart, s->resid, s->o.tol, s->d_nactive, s->st));
  return LAPH_OK;
}

// Step n (1-based) of a filter pass; fin: the pass's last step (writes W); nos: every active problem runs
// the pass directly, so steps past the second read no S.
static int filter_step(laph_solver* s, int n, bool fin, bool nos, cudaStream_t st) {
  const int bf = s->o.link_prec == LAPH_LINKS_BF16;
  const void* links = bf ? s->Ubf : static_cast<const void*>(s->Uf32);
  const float2* X = (n == 1) ? s->S : s->E[(n - 2) % 3];
  const float2* Z = (n >= 3) ? s->E[(n - 3) % 3] : nullptr;
  float2* Yo = s->E[(n - 1) % 3];
  return cheb_step(s->d_pd, s->d_ps, s->st_filt, s->np, s->nb_filt, s->kb, bf, links, s->scale, X, Z, s->S, Yo, s->V,
                   s->W, s->tcoef, n, fin, s->fvariant, s->tile, s->lmax, s->d_ferr, nos && n >= 3, st);
}

static int filter(laph_solver* s, int m, bool nos) {
  LAPH_TRY(coef(s->d_pd, s->d_ps, s->np, s->theta, s->tcoef, s->scol, m, nullptr, s->st));
  LAPH_TRY(direct_start(s->d_pd, s->d_ps, s->st_filt, s->np, s->nb_filt, s->kb, s->tile, s->V, s->S, s->st));
  for (int n = 1; n < m; ++n) LAPH_TRY(filter_step(s, n, n == m - 1, nos, s->st));
  return LAPH_OK;
}

}  // extern "C"

// Capture `body` on the solver's stream into an executable graph.
template <typename F>
static int capture(laph_solver* s, cudaGraphExec_t* exec, F body) {
  LAPH_CUDA_TRY(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
  const int rc = body();
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s->st, &g);
  if (rc != LAPH_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) {
    set_error("graph capture failed: %s", cudaGetErrorString(e));
    return LAPH_ECUDA;
  }
  const cudaError_t ei = cudaGraphInstantiate(exec, g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) {
    set_error("graph instantiation failed: %s", cudaGetErrorString(ei));
    return LAPH_ECUDA;
  }
  return LAPH_OK;
}

static int filter_graph(laph_solver* s, int m, bool nos) {
  const int key = 2 * m + (nos ? 1 : 0);
  auto it = s->g_filter.find(key);
  if (it == s->g_filter.end()) {
    cudaGraphExec_t ex = nullptr;
    LAPH_TRY(capture(s, &ex, [&] { return filter(s, m, nos); }));
    it = s->g_filter.emplace(key, ex).first;
  }
  LAPH_CUDA_TRY(cudaGraphLaunch(it->second, s->st));
  return LAPH_OK;
}

static int rr_graph(laph_solver* s) {
  if (!s->g_rr) LAPH_TRY(capture(s, &s->g_rr, [&] { return iteration_rr(s, 0); }));
  LAPH_CUDA_TRY(cudaGraphLaunch(s->g_rr, s->st));
  return LAPH_OK;
}

// Everything a solve does before its first outer iteration: the pristine links
// into the working copy, smearing, the filter links, the start state, the
// features and the window (learned, Lanczos or fixed), the start block and its
// residuals.  Queued on the solver's stream; counts its kernels in *nlaunch.
static int solve_setup(laph_solver* s, bool device_loop, long long* nlaunch_out) {
  const laph_solve_opts& o = s->o;
  long long nlaunch = 0;
  LAPH_CUDA_TRY(cudaMemcpyAsync(s->U64, s->U64raw, s->hd.back().u64 * sizeof(double2) + 27 * sizeof(double2) * s->hd.back().V3,
                                cudaMemcpyDeviceToDevice, s->st));
  // smearing, per run of consecutive problems with equal L and parameters
  for (int i = 0; i < s->np;) {
    int j = i;
    while (j < s->np && s->hd[j].L == s->hd[i].L && s->sp1[j] == s->sp1[i] && s->sp2[j] == s->sp2[i]) ++j;
    LAPH_TRY(smear_batch(s->U64 + s->hd[i].u64, s->Utmp, s->dec, s->hd[i].L, j - i, o.smear_kind, s->sp1[i],
                         s->sp2[i], o.smear_iters, o.smear_compat, s->st));
    if (o.smear_kind != LAPH_SMEAR_NONE) nlaunch += (long long)o.smear_iters * (o.smear_kind == LAPH_SMEAR_HYP ? 2 : 1);
    i = j;
  }
  LAPH_TRY(pack_links(s->d_pd, s->st_site, s->np, s->nb_site, s->U64, s->Uf32, s->Ubf, s->scale,
                      o.link_prec == LAPH_LINKS_BF16, s->st));
  // initial state (lam_max = 12 or the fixed one, lam_cut, all active)
  LAPH_CUDA_TRY(cudaMemcpyAsync(s->d_ps, s->d_ps0, s->np * sizeof(ProbState), cudaMemcpyDeviceToDevice, s->st));
  // per-timeslice features (plaquette moments + 10-step Lanczos); the learned
  // window sets the first pass's lam_cut and degree from them
  s->deg0 = 0;
  if (o.window != LAPH_WINDOW_FIXED) {
    for (int i = 0; i < s->np;) {
      int j = i;
      while (j < s->np && s->hd[j].L == s->hd[i].L) ++j;
      LAPH_TRY(plaquette_moments_batch(s->U64 + s->hd[i].u64, s->hd[i].L, j - i, s->plaq + 4 * (size_t)i, s->st));
      i = j;
    }
    LAPH_TRY(features(s->d_pd, s->np, s->U64, s->plaq, s->W, s->feats, s->bound, s->st));
    nlaunch += 2;
    if (o.window == LAPH_WINDOW_MLP) {
      const double margin = o.window_margin > 0.0 ? o.window_margin : kWindowMargin;
      LAPH_TRY(window_infer(s->d_pd, s->d_ps, s->np, s->feats, s->model, s->mwork, s->bound, s->wdeg, margin,
                            s->st));
      if (!device_loop) {  // the device-side loop takes the largest degree on the device
        std::vector<int> dg(s->np);
        LAPH_CUDA_TRY(cudaMemcpyAsync(dg.data(), s->wdeg, s->np * sizeof(int), cudaMemcpyDeviceToHost, s->st));
        LAPH_CUDA_TRY(cudaStreamSynchronize(s->st));
        for (int d : dg) s->deg0 = std::max(s->deg0, d);
      }
      nlaunch += 3;
    }
  }
  // With the window known before any Ritz value (learned or fixed), the random
  // block goes straight into the first filter pass; otherwise a first
  // Rayleigh-Ritz of the random block sets the window.
  const bool window_known = o.window == LAPH_WINDOW_MLP || (o.window == LAPH_WINDOW_FIXED && o.lam_cut > 0.0);
  if (window_known) {
    LAPH_TRY(random_block(s->d_pd, s->st_rand, s->np, s->nb_rand, s->V, o.seed, s->st));
    if (!device_loop) LAPH_CUDA_TRY(cudaEventRecord(s->ev1, s->st));
    LAPH_TRY(start_window(s->d_pd, s->d_ps, s->np, s->theta, s->st));
    LAPH_TRY(residual(s));
    LAPH_TRY(zero_int(s->d_nactive, s->st));
    LAPH_TRY(resid_check(s->d_pd, s->d_ps, s->np, s->rpart, s->resid, s->o.tol, s->d_nactive, s->st));
    nlaunch += 2 + 5;  // pack, random block, window state, residual, zero, check
  } else {
    LAPH_TRY(random_block(s->d_pd, s->st_rand, s->np, s->nb_rand, s->W, o.seed, s->st));
    if (!device_loop) LAPH_CUDA_TRY(cudaEventRecord(s->ev1, s->st));
    LAPH_TRY(iteration_rr(s, 1));
    nlaunch += 2 + 8;  // pack, random block, first Rayleigh-Ritz
  }
  *nlaunch_out = nlaunch;
  return LAPH_OK;
}

// Per-problem results of the last run from the host copy of the states.
static int fill_results(laph_solver* s, laph_result* res) {
  const laph_solve_opts& o = s->o;
  int status = LAPH_OK;
  if (s->fvariant == 3) {
    int ferr = 0;
    if (cudaMemcpy(&ferr, s->d_ferr, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return LAPH_ECUDA;
    if (ferr != 0) {
      set_error("laph_solver_run: the staged filter's copy pipeline failed (code %d); results are invalid", ferr);
      return LAPH_ECUDA;
    }
  }
  for (int i = 0; i < s->np; ++i) {
    const ProbState& p = s->hps[i];
    if (p.active) status = LAPH_ENOTCONV;
    if (res) {
      laph_result& r = res[i];
      r.status = p.active ? LAPH_ENOTCONV : LAPH_OK;
      r.iters = p.iters;
      r.nconv = p.nconv;
      r.deg = s->mdeg;
      r.lam_cut0 = o.lam_cut;
      r.lam_max = s->lam_max0[i];
      r.window_fallback = s->fallback[i];
      r.max_resid = p.max_resid;
      std::vector<double> nv(s->hd[i].nev);
      cudaMemcpy(nv.data(), s->norms + s->hd[i].kv, nv.size() * sizeof(double), cudaMemcpyDeviceToHost);
      double tr = 0.0;
      for (double v : nv) tr += v;
      r.trace_vdv = tr;
    }
  }
  if (status != LAPH_OK) set_error("laph_solver_run: max_it = %d reached before all problems converged", o.max_it);
  return status;
}

// ------------------------------------------------------ device-side loop ---
// The whole solve as one executable graph:
//   setup (solve_setup) -> loop_init -> loop_cond
//   WHILE (any problem active and it < max_it):
//       loop_pass_begin (degree, the learned window's check, counters, step switches)
//       coef (degree read on the device)
//       SWITCH per filter step n = 1..mdeg-1: {plain step n | last step n | nothing}
//       loop_pass_end, Rayleigh-Ritz + residuals + convergence mask, loop_cond
//   loop_end -> phase fix
// so no host round trip separates the passes (the host loop reads the mask
// once per pass).  Built by stream capture into the graph and its bodies.

// Capture `body` on the solver's stream into `g` after the nodes `deps`;
// on return `deps` holds the leaf nodes of the capture.
template <typename F>
static int capture_into(laph_solver* s, cudaGraph_t g, std::vector<cudaGraphNode_t>& deps, F body) {
  LAPH_CUDA_TRY(cudaStreamBeginCaptureToGraph(s->st, g, deps.empty() ? nullptr : deps.data(), nullptr, deps.size(),
                                              cudaStreamCaptureModeThreadLocal));
  int rc = body();
  if (rc == LAPH_OK) {
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* d = nullptr;
    size_t nd = 0;
    const cudaError_t e = cudaStreamGetCaptureInfo(s->st, &cs, nullptr, nullptr, &d, &nd);
    if (e != cudaSuccess || cs != cudaStreamCaptureStatusActive) {
      set_error("graph capture: %s", cudaGetErrorString(e));
      rc = LAPH_ECUDA;
    } else {
      deps.assign(d, d + nd);
    }
  }
  cudaGraph_t out = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s->st, &out);
  if (rc == LAPH_OK && e != cudaSuccess) {
    set_error("graph capture: %s", cudaGetErrorString(e));
    rc = LAPH_ECUDA;
  }
  return rc;
}

// A conditional node after `deps` in g; its body graphs go to bodies[0..size).
static int add_conditional(cudaGraph_t g, std::vector<cudaGraphNode_t>& deps, cudaGraphConditionalHandle h,
                           cudaGraphConditionalNodeType type, unsigned size, cudaGraph_t* bodies) {
  cudaGraphNodeParams np{};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = type;
  np.conditional.size = size;
  cudaGraphNode_t node;
  LAPH_CUDA_TRY(cudaGraphAddNode(&node, g, deps.empty() ? nullptr : deps.data(), deps.size(), &np));
  for (unsigned i = 0; i < size; ++i) bodies[i] = np.conditional.phGraph_out[i];
  deps.assign(1, node);
  return LAPH_OK;
}

static int build_solve_graph(laph_solver* s) {
  const laph_solve_opts& o = s->o;
  cudaGraph_t g = nullptr;
  LAPH_CUDA_TRY(cudaGraphCreate(&g, 0));
  auto done = [&](int rc) {
    cudaGraphDestroy(g);
    return rc;
  };
  cudaGraphConditionalHandle h_loop;
  if (cudaGraphConditionalHandleCreate(&h_loop, g, 0, 0) != cudaSuccess) {
    set_error("conditional graph nodes not available");
    return done(LAPH_ECUDA);
  }
  LoopParams lp{};
  lp.mdeg = s->mdeg;
  lp.max_it = o.max_it;
  lp.kb = s->kb;
  lp.mlp = o.window == LAPH_WINDOW_MLP;
  lp.lbytes = o.link_prec == LAPH_LINKS_BF16 ? 112.0 : 216.0;
  lp.lam_top = o.lam_max > 0.0 ? o.lam_max : 12.0;
  lp.cap_resid = kCapResid;
  lp.win_check = kWindowCheck;
  lp.direct_resid = direct_resid(o);
  long long nsetup = 0;
  std::vector<cudaGraphNode_t> deps;
  int rc = capture_into(s, g, deps, [&]() -> int {
    LAPH_TRY(loop_stamp(&s->ls->t_start, s->st));
    LAPH_TRY(solve_setup(s, true, &nsetup));
    LAPH_CUDA_TRY(cudaMemsetAsync(s->d_fallback, 0, sizeof(int) * s->np, s->st));
    LAPH_TRY(loop_init(s->ls, o.window == LAPH_WINDOW_MLP ? s->wdeg : nullptr, s->np, s->st));
    return loop_cond(s->ls, s->d_nactive, o.max_it, h_loop, s->st);
  });
  if (rc != LAPH_OK) return done(rc);
  cudaGraph_t body;
  if ((rc = add_conditional(g, deps, h_loop, cudaGraphCondTypeWhile, 1, &body)) != LAPH_OK) return done(rc);
  std::vector<cudaGraphNode_t> top = deps;  // the WHILE node
  // the pass: one SWITCH handle per filter step position
  std::vector<cudaGraphConditionalHandle> hs(s->mdeg + 1, 0);
  for (int n = 1; n < s->mdeg; ++n)
    if (cudaGraphConditionalHandleCreate(&hs[n], body, 4, 0) != cudaSuccess) {
      set_error("conditional graph nodes not available");
      return done(LAPH_ECUDA);
    }
  if (cudaMemcpy(s->d_steps, hs.data(), hs.size() * sizeof(hs[0]), cudaMemcpyHostToDevice) != cudaSuccess)
    return done(LAPH_ECUDA);
  std::vector<cudaGraphNode_t> bd;
  rc = capture_into(s, body, bd, [&]() -> int {
    LAPH_TRY(loop_pass_begin(s->d_pd, s->d_ps, s->np, s->ls, s->d_degs, s->d_lam_max0, s->d_fallback, s->d_steps,
                             lp, s->st));
    LAPH_TRY(coef(s->d_pd, s->d_ps, s->np, s->theta, s->tcoef, s->scol, 0, &s->ls->m, s->st));
    return direct_start(s->d_pd, s->d_ps, s->st_filt, s->np, s->nb_filt, s->kb, s->tile, s->V, s->S, s->st);
  });
  if (rc != LAPH_OK) return done(rc);
  // SWITCH per step position: middle / last step, and for n >= 3 the same two without S
  for (int n = 1; n < s->mdeg; ++n) {
    const unsigned nb = n >= 3 ? 4u : 2u;
    cudaGraph_t b[4];
    if ((rc = add_conditional(body, bd, hs[n], cudaGraphCondTypeSwitch, nb, b)) != LAPH_OK) return done(rc);
    for (unsigned br = 0; br < nb; ++br) {
      std::vector<cudaGraphNode_t> none;
      if ((rc = capture_into(s, b[br], none,
                             [&]() -> int { return filter_step(s, n, (br & 1u) != 0, br >= 2, s->st); })) != LAPH_OK)
        return done(rc);
    }
  }
  rc = capture_into(s, body, bd, [&]() -> int {
    LAPH_TRY(loop_pass_end(s->ls, s->st));
    LAPH_TRY(iteration_rr(s, 0));
    return loop_cond(s->ls, s->d_nactive, o.max_it, h_loop, s->st);
  });
  if (rc != LAPH_OK) return done(rc);
  rc = capture_into(s, g, top, [&]() -> int {
    LAPH_TRY(loop_end(s->ls, s->st));
    return phase_fix(s->d_pd, s->st_col, s->np, s->nb_col, s->V, s->phases, s->norms, o.phase_fix, s->st);
  });
  if (rc != LAPH_OK) return done(rc);
  const cudaError_t ei = cudaGraphInstantiate(&s->g_solve, g, 0);
  if (ei != cudaSuccess) {
    s->g_solve = nullptr;
    set_error("solve graph instantiation failed: %s", cudaGetErrorString(ei));
    return done(LAPH_ECUDA);
  }
  // kernels outside the loop: stamp, setup, loop_init, loop_cond, loop_end, phase fix
  s->solve_setup_launches = 1 + nsetup + 2 + 2;
  return done(LAPH_OK);
}

static int run_device_loop(laph_solver* s, laph_result* res) {
  LAPH_CUDA_TRY(cudaEventRecord(s->ev0, s->st));
  LAPH_CUDA_TRY(cudaGraphLaunch(s->g_solve, s->st));
  LAPH_CUDA_TRY(cudaEventRecord(s->ev2, s->st));
  LoopState ls;
  LAPH_CUDA_TRY(cudaMemcpyAsync(&ls, s->ls, sizeof ls, cudaMemcpyDeviceToHost, s->st));
  LAPH_CUDA_TRY(cudaMemcpyAsync(s->hps.data(), s->d_ps, s->np * sizeof(ProbState), cudaMemcpyDeviceToHost, s->st));
  s->lam_max0.assign(s->np, 0.0);
  s->fallback.assign(s->np, 0);
  LAPH_CUDA_TRY(cudaMemcpyAsync(s->lam_max0.data(), s->d_lam_max0, s->np * sizeof(double), cudaMemcpyDeviceToHost,
                                s->st));
  LAPH_CUDA_TRY(cudaMemcpyAsync(s->fallback.data(), s->d_fallback, s->np * sizeof(int), cudaMemcpyDeviceToHost, s->st));
  LAPH_CUDA_TRY(cudaStreamSynchronize(s->st));
  s->degs.assign(std::max(ls.npass, 0), 0);
  if (ls.npass > 0)
    LAPH_CUDA_TRY(cudaMemcpy(s->degs.data(), s->d_degs, ls.npass * sizeof(int), cudaMemcpyDeviceToHost));
  float b = 0.f;
  cudaEventElapsedTime(&b, s->ev0, s->ev2);
  s->ms[0] = 1e-6 * (double)(ls.t_loop - ls.t_start);
  s->ms[1] = 1e-6 * ls.filt_ns;
  s->ms[3] = b;
  s->ms[2] = b - s->ms[0] - s->ms[1];
  long long fl = 0;
  for (int m : s->degs) fl += m - 1;
  s->cnt[0] = (long long)ls.sv_steps;
  s->cnt[1] = fl;
  // per pass: loop_pass_begin, coef, direct_start, the m - 1 steps, loop_pass_end, 8 Rayleigh-Ritz kernels,
  // loop_cond
  s->cnt[2] = s->solve_setup_launches + 13LL * ls.npass + fl;
  s->fbytes[0] = ls.fbytes[0];
  s->fbytes[1] = ls.fbytes[1];
  s->ran = 1;
  s->last_loop = 1;
  s->last_graph_launches = 1;
  return fill_results(s, res);
}
extern "C" {

int laph_solver_run(laph_solver* s, laph_result* res) {
  if (!s) {
    set_error("null solver");
    return LAPH_EINVAL;
  }
  for (int i = 0; i < s->np; ++i)
    if (!s->links_set[i]) {
      set_error("laph_solver_run: links of problem %d not set", i);
      return LAPH_EINVAL;
    }
  LAPH_CUDA_TRY(cudaSetDevice(s->dev));
  const laph_solve_opts& o = s->o;
  if (o.window == LAPH_WINDOW_MLP && !s->have_model) {
    set_error("laph_solver_run: window = MLP but no model set (laph_solver_set_window_model)");
    return LAPH_EINVAL;
  }
  if (s->conv_pending) {  // asynchronous read-backs still converting V: let them finish reading it
    LAPH_CUDA_TRY(cudaStreamWaitEvent(s->st, s->ev_conv, 0));
    s->conv_pending = 0;
  }
  const char* tr_env = std::getenv("LAPH_TRACE");
  const bool trace = tr_env && *tr_env && *tr_env != '0';
  if (!trace && !o.host_loop && !s->solve_graph_failed) {
    if (!s->g_solve && build_solve_graph(s) != LAPH_OK) {
      // conditional graph nodes refused (driver or runtime too old): the host loop from here on
      s->solve_graph_failed = 1;
      cudaGetLastError();
    }
    if (s->g_solve) return run_device_loop(s, res);
  }
  LAPH_CUDA_TRY(cudaEventRecord(s->ev0, s->st));
  long long nlaunch = 0;
  LAPH_TRY(solve_setup(s, false, &nlaunch));
  s->cnt[0] = s->cnt[1] = s->cnt[2] = 0;
  s->fbytes[0] = s->fbytes[1] = 0.0;
  s->fallback.assign(s->np, 0);
  s->lam_max0.assign(s->np, 0.0);
  s->degs.clear();
  double filt_ms = 0.0;
  if (s->evf.empty()) {
    s->evf.resize(2);
    cudaEventCreate(&s->evf[0]);
    cudaEventCreate(&s->evf[1]);
  }
  if (trace) LAPH_CUDA_TRY(cudaMemsetAsync(s->tstamp, 0, (size_t)s->np * kSmallPhases * sizeof(unsigned long long), s->st));
  int it = 1;
  for (; it < o.max_it; ++it) {
    LAPH_CUDA_TRY(cudaMemcpyAsync(s->h_nactive, s->d_nactive, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    LAPH_CUDA_TRY(cudaMemcpyAsync(s->hps.data(), s->d_ps, s->np * sizeof(ProbState), cudaMemcpyDeviceToHost, s->st));
    LAPH_CUDA_TRY(cudaStreamSynchronize(s->st));
    if (trace) {
      // LAPH_TRACE=1: one line per outer iteration with the batch's state after the last Rayleigh-Ritz
      long long nl = 0, nk = 0, nc = 0, nv = 0;
      double mr = 0.0;
      for (int i = 0; i < s->np; ++i) {
        nl += s->hps[i].nlock;
        nk += s->hd[i].k;
        nc += s->hps[i].nconv;
        nv += s->hd[i].nev;
        if (s->hps[i].active) mr = std::max(mr, s->hps[i].max_resid);
      }
      std::fprintf(stderr, "laph_trace it %d active %d locked %lld/%lld converged %lld/%lld max_resid %.3e\n", it,
                   *s->h_nactive, nl, nk, nc, nv, mr);
      // mean duration of the phases of the last small dense step over the problems that ran it
      std::vector<unsigned long long> ts((size_t)s->np * kSmallPhases);
      if (cudaMemcpy(ts.data(), s->tstamp, ts.size() * sizeof(ts[0]), cudaMemcpyDeviceToHost) == cudaSuccess) {
        double ph[kSmallPhases - 1] = {0};
        int cnt = 0;
        for (int i = 0; i < s->np; ++i) {
          const unsigned long long* t = &ts[(size_t)i * kSmallPhases];
          if (t[0] == 0 || t[kSmallPhases - 1] < t[0]) continue;
          ++cnt;
          for (int q = 0; q + 1 < kSmallPhases; ++q) ph[q] += 1e-3 * (double)(t[q + 1] - t[q]);
        }
        cudaMemset(s->tstamp, 0, ts.size() * sizeof(ts[0]));
        if (cnt)
          std::fprintf(stderr,
                       "laph_trace it %d small dense us: cholesky %.0f inverse %.0f project %.0f jacobi %.0f "
                       "sort+C %.0f window %.0f\n",
                       it, ph[0] / cnt, ph[1] / cnt, ph[2] / cnt, ph[3] / cnt, ph[4] / cnt, ph[5] / cnt);
      }
    }
    if (it == 1) {
      s->lam_max0.resize(s->np);
      for (int i = 0; i < s->np; ++i) s->lam_max0[i] = s->hps[i].lam_max;
    }
    // The learned window's check, after its first pass and Rayleigh-Ritz: a
    // problem whose wanted residuals did not fall below kWindowCheck, whose
    // Cholesky needed a clamped pivot or whose state is not finite goes on as
    // the non-learned method would (lam_max back to the exact bound 12, the
    // cut from its Ritz values).
    if (it == 2 && o.window == LAPH_WINDOW_MLP) {
      bool any = false;
      for (int i = 0; i < s->np; ++i) {
        ProbState& p = s->hps[i];
        if (!p.active || (p.max_resid < kWindowCheck && !p.chol_fail && std::isfinite(p.lam_cut))) continue;
        s->fallback[i] = 1;
        any = true;
        const double top = o.lam_max > 0.0 ? o.lam_max : 12.0;
        if (!(p.lam_max < top) && std::isfinite(p.lam_cut)) continue;  // window already the non-learned one
        p.lam_max = top;
        double cut = std::isfinite(p.lam_cut) ? p.lam_cut : 0.5 * top;
        cut = std::min(std::max(cut, 1e-6), top - 1e-3);
        p.lam_cut = cut;
        p.c_hop = 2.0 / (top - cut);
        p.c_diag = (top + cut - 12.0) / (top - cut);
      }
      if (any)
        LAPH_CUDA_TRY(cudaMemcpyAsync(s->d_ps, s->hps.data(), s->np * sizeof(ProbState), cudaMemcpyHostToDevice, s->st));
    }
    if (*s->h_nactive == 0) break;
    // Degree of this pass.  While the Ritz vectors are still poor (largest
    // wanted residual > 1e-2) the amplification of the filter is capped at
    // 1e6 relative to the damped interval -- taken at lambda = 0, the bottom
    // of the spectrum of -Delta -- so the filtered block cannot collapse onto
    // the lowest eigenvectors and break the Cholesky QR; afterwards the
    // correction form keeps the block well conditioned at any degree.
    int m = s->mdeg;
    if (it == 1 && s->deg0 > 0) m = std::min(m, std::max(2, s->deg0));
    for (int i = 0; i < s->np; ++i) {
      const ProbState& p = s->hps[i];
      if (!p.active || !(p.max_resid > kCapResid)) continue;
      const double tb0 = 1.0 + 2.0 * p.lam_cut / (p.lam_max - p.lam_cut);
      // (1e8 after the first pass: 34 instead of 26 in pass 2, same 8 iterations, no faster; 1e10: 42, slower)
      const double ratio = std::acosh(1e6) / std::acosh(std::max(tb0, 1.0 + 1e-12));
      const int m_safe = std::isfinite(ratio) ? (int)std::min(std::floor(ratio), 1e6) : 2;  // NaN window: degree 2
      m = std::min(m, std::max(2, m_safe));
    }
    // Direct passes: a problem whose largest wanted residual is above direct_resid filters V itself in FP32
    // this pass (the device loop's rule, k_loop_pass_begin); when every active problem does, the steps past
    // the second read no S.
    int nact_p = 0, ndir_p = 0;
    const double dres = direct_resid(o);
    for (int i = 0; i < s->np; ++i) {
      ProbState& p = s->hps[i];
      if (p.active) {
        if (p.direct && !(p.max_resid < 0.5 * p.resid_begin)) p.direct_off = 1;
        p.resid_begin = p.max_resid;
      }
      p.direct = p.active && !p.direct_off && dres >= 0.0 && !(p.max_resid <= dres) ? 1 : 0;
      nact_p += p.active ? 1 : 0;
      ndir_p += p.direct;
    }
    const bool nos = nact_p > 0 && ndir_p == nact_p;
    LAPH_CUDA_TRY(cudaMemcpyAsync(s->d_ps, s->hps.data(), s->np * sizeof(ProbState), cudaMemcpyHostToDevice, s->st));
    const double lbytes = s->o.link_prec == LAPH_LINKS_BF16 ? 112.0 : 216.0;  // per site per column block
    for (int i = 0; i < s->np; ++i) {
      if (!s->hps[i].active) continue;
      const ProbDesc& d = s->hd[i];
      const int nl = s->hps[i].nlock, nact = d.k - nl;
      s->cnt[0] += (long long)d.V3 * nact * (m - 1);
      const int nblk = (d.k + s->kb - 1) / s->kb - nl / s->kb;  // column blocks with an unlocked column
      double per = s->hps[i].direct ? 72.0 : 0.0;  // bytes per unlocked site-vector over the pass
      for (int n = 1; n < m; ++n) {
        const int reads = n == 1 ? 1 : (n == 2 ? 2 : (nos ? 2 : 3));
        per += reads * 24.0 + (n == m - 1 ? 96.0 : 24.0);
      }
      s->fbytes[0] += (double)d.V3 * (nact * per + nl * 96.0 + (double)nblk * (m - 1) * lbytes);
      s->fbytes[1] += (double)d.V3 * (m - 1) * (nact * 72.0 + (double)nblk * lbytes);
    }
    s->cnt[1] += m - 1;
    s->degs.push_back(m);
    if (trace) std::fprintf(stderr, "laph_trace it %d filter degree %d direct %d/%d\n", it, m, ndir_p, nact_p);
    LAPH_CUDA_TRY(cudaEventRecord(s->evf[0], s->st));
    LAPH_TRY(filter_graph(s, m, nos));
    LAPH_CUDA_TRY(cudaEventRecord(s->evf[1], s->st));
    LAPH_TRY(rr_graph(s));
    nlaunch += 2 + (m - 1) + 8;
    float f = 0.f;
    LAPH_CUDA_TRY(cudaEventSynchronize(s->evf[1]));
    LAPH_CUDA_TRY(cudaEventElapsedTime(&f, s->evf[0], s->evf[1]));
    filt_ms += f;
  }
  LAPH_TRY(phase_fix(s->d_pd, s->st_col, s->np, s->nb_col, s->V, s->phases, s->norms, o.phase_fix, s->st));
  s->cnt[2] = nlaunch + 1;
  LAPH_CUDA_TRY(cudaEventRecord(s->ev2, s->st));
  LAPH_CUDA_TRY(cudaMemcpyAsync(s->hps.data(), s->d_ps, s->np * sizeof(ProbState), cudaMemcpyDeviceToHost, s->st));
  LAPH_CUDA_TRY(cudaStreamSynchronize(s->st));
  float a = 0.f, b = 0.f;
  cudaEventElapsedTime(&a, s->ev0, s->ev1);
  cudaEventElapsedTime(&b, s->ev0, s->ev2);
  s->ms[0] = a;
  s->ms[1] = filt_ms;
  s->ms[3] = b;
  s->ms[2] = b - a - filt_ms;
  s->ran = 1;
  s->last_loop = 0;
  s->last_graph_launches = 2LL * (long long)s->degs.size();
  return fill_results(s, res);
}

int laph_solver_get(laph_solver* s, int i, double* evals, double* evecs, double* phases, int on_device) {
  if (!s || i < 0 || i >= s->np || !s->ran) {
    set_error("laph_solver_get: bad argument or solver not run");
    return LAPH_EINVAL;
  }
  LAPH_CUDA_TRY(cudaSetDevice(s->dev));
  const ProbDesc& d = s->hd[i];
  const cudaMemcpyKind kd = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (evals) {
    std::vector<double> th(d.nev);
    LAPH_CUDA_TRY(cudaMemcpyAsync(th.data(), s->theta + d.kv, d.nev * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    LAPH_CUDA_TRY(cudaStreamSynchronize(s->st));
    for (auto& v : th) v = -v;  // eigenvalues of Delta (recover_spectrum convention)
    LAPH_CUDA_TRY(cudaMemcpy(evals, th.data(), d.nev * sizeof(double), on_device ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost));
  }
  if (evecs) {
    // the block is colour-major on the device; the caller gets 3*site + colour
    if (on_device) {
      LAPH_TRY(to_reference(s->V + d.blk, reinterpret_cast<double2*>(evecs), d.V3, d.nev, s->st));
    } else {
      LAPH_TRY(to_reference(s->V + d.blk, s->W + d.blk, d.V3, d.nev, s->st));
      LAPH_CUDA_TRY(cudaMemcpyAsync(evecs, s->W + d.blk, (size_t)d.dim * d.nev * sizeof(double2), kd, s->st));
    }
  }
  if (phases) LAPH_CUDA_TRY(cudaMemcpyAsync(phases, s->phases + d.kv, d.nev * sizeof(double), kd, s->st));
  LAPH_CUDA_TRY(cudaStreamSynchronize(s->st));
  return LAPH_OK;
}

// Negate the Ritz values of one problem into the staging pool (the
// eigenvalues of Delta, recover_spectrum's sign) and copy its phases beside them.
__global__ void k_out_vals(const double* __restrict__ theta, const double* __restrict__ phases, int nev,
                           double* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nev) return;
  out[j] = -theta[j];
  out[nev + j] = phases[j];
}

int laph_solver_get_async(laph_solver* s, int i, double* evals, double* evecs, double* phases) {
  if (!s || i < 0 || i >= s->np || !s->ran) {
    set_error("laph_solver_get_async: bad argument or solver not run");
    return LAPH_EINVAL;
  }
  LAPH_CUDA_TRY(cudaSetDevice(s->dev));
  if (!s->st_out) {
    size_t nvec = 0, nval = 0;
    s->out_off.resize(s->np);
    s->out_voff.resize(s->np);
    for (int p = 0; p < s->np; ++p) {
      s->out_off[p] = nvec;
      s->out_voff[p] = nval;
      nvec += (size_t)s->hd[p].dim * s->hd[p].nev;
      nval += 2 * (size_t)s->hd[p].nev;
    }
    bool ok = cudaStreamCreateWithFlags(&s->st_out, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&s->st_conv, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&s->ev_run, cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&s->ev_conv, cudaEventDisableTiming) == cudaSuccess &&
              cudaMalloc(&s->out_vec, sizeof(double2) * nvec) == cudaSuccess &&
              cudaMalloc(&s->out_val, sizeof(double) * nval) == cudaSuccess;
    s->ev_ready.assign(s->np, nullptr);
    s->ev_copied.assign(s->np, nullptr);
    s->copied_rec.assign(s->np, 0);
    for (int p = 0; p < s->np && ok; ++p)
      ok = cudaEventCreateWithFlags(&s->ev_ready[p], cudaEventDisableTiming) == cudaSuccess &&
           cudaEventCreateWithFlags(&s->ev_copied[p], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      set_error("laph_solver_get_async: cannot set up the read-back streams and the %zu-byte staging pool",
                sizeof(double2) * nvec);
      return LAPH_ENOMEM;
    }
  }
  const ProbDesc& d = s->hd[i];
  double2* ov = s->out_vec + s->out_off[i];
  double* oval = s->out_val + s->out_voff[i];
  // conversion stream: after everything queued on the compute stream so far (the
  // run), and after the previous read-back of this problem's staging left it
  LAPH_CUDA_TRY(cudaEventRecord(s->ev_run, s->st));
  LAPH_CUDA_TRY(cudaStreamWaitEvent(s->st_conv, s->ev_run, 0));
  if (s->copied_rec[i]) LAPH_CUDA_TRY(cudaStreamWaitEvent(s->st_conv, s->ev_copied[i], 0));
  if (evecs) LAPH_TRY(to_reference(s->V + d.blk, ov, d.V3, d.nev, s->st_conv));
  k_out_vals<<<ceil_div(d.nev, 128), 128, 0, s->st_conv>>>(s->theta + d.kv, s->phases + d.kv, d.nev, oval);
  LAPH_CUDA_TRY(cudaGetLastError());
  LAPH_CUDA_TRY(cudaEventRecord(s->ev_ready[i], s->st_conv));
  LAPH_CUDA_TRY(cudaEventRecord(s->ev_conv, s->st_conv));  // the next run waits for this (conversions only)
  s->conv_pending = 1;
  // copy stream: staging -> host once converted
  LAPH_CUDA_TRY(cudaStreamWaitEvent(s->st_out, s->ev_ready[i], 0));
  if (evecs)
    LAPH_CUDA_TRY(cudaMemcpyAsync(evecs, ov, sizeof(double2) * d.dim * d.nev, cudaMemcpyDeviceToHost, s->st_out));
  if (evals) LAPH_CUDA_TRY(cudaMemcpyAsync(evals, oval, sizeof(double) * d.nev, cudaMemcpyDeviceToHost, s->st_out));
  if (phases)
    LAPH_CUDA_TRY(cudaMemcpyAsync(phases, oval + d.nev, sizeof(double) * d.nev, cudaMemcpyDeviceToHost, s->st_out));
  LAPH_CUDA_TRY(cudaEventRecord(s->ev_copied[i], s->st_out));
  s->copied_rec[i] = 1;
  return LAPH_OK;
}

int laph_solver_wait(laph_solver* s) {
  if (!s) {
    set_error("laph_solver_wait: null solver");
    return LAPH_EINVAL;
  }
  if (!s->st_out) return LAPH_OK;
  LAPH_CUDA_TRY(cudaSetDevice(s->dev));
  LAPH_CUDA_TRY(cudaStreamSynchronize(s->st_conv));
  LAPH_CUDA_TRY(cudaStreamSynchronize(s->st_out));
  return LAPH_OK;
}

int laph_solver_set_window_model(laph_solver* s, const float* model, int nfloats) {
  if (!s || !model || nfloats != kMlpParams + kMlpNorm) {
    set_error("laph_solver_set_window_model: need %d floats (parameters + normalisation)", kMlpParams + kMlpNorm);
    return LAPH_EINVAL;
  }
  LAPH_CUDA_TRY(cudaSetDevice(s->dev));
  LAPH_CUDA_TRY(cudaMemcpyAsync(s->model, model, sizeof(float) * nfloats, cudaMemcpyHostToDevice, s->st));
  LAPH_CUDA_TRY(cudaStreamSynchronize(s->st));
  s->have_model = 1;
  return LAPH_OK;
}

int laph_solver_features(laph_solver* s, float* feats, double* bound) {
  if (!s || !s->ran) {
    set_error("laph_solver_features: solver not run");
    return LAPH_EINVAL;
  }
  LAPH_CUDA_TRY(cudaSetDevice(s->dev));
  if (feats)
    LAPH_CUDA_TRY(cudaMemcpyAsync(feats, s->feats, sizeof(float) * kMlpIn * s->np, cudaMemcpyDeviceToHost, s->st));
  if (bound) LAPH_CUDA_TRY(cudaMemcpyAsync(bound, s->bound, sizeof(double) * s->np, cudaMemcpyDeviceToHost, s->st));
  LAPH_CUDA_TRY(cudaStreamSynchronize(s->st));
  return LAPH_OK;
}

int laph_solver_ritz(laph_solver* s, int i, double* theta, int* k) {
  if (!s || !s->ran || i < 0 || i >= s->np || !theta) {
    set_error("laph_solver_ritz: bad argument or solver not run");
    return LAPH_EINVAL;
  }
  LAPH_CUDA_TRY(cudaSetDevice(s->dev));
  const ProbDesc& d = s->hd[i];
  LAPH_CUDA_TRY(cudaMemcpyAsync(theta, s->theta + d.kv, sizeof(double) * d.k, cudaMemcpyDeviceToHost, s->st));
  LAPH_CUDA_TRY(cudaStreamSynchronize(s->st));
  if (k) *k = d.k;
  return LAPH_OK;
}

int laph_solver_stream(laph_solver* s, void** stream) {
  if (!s || !stream) {
    set_error("laph_solver_stream: bad argument");
    return LAPH_EINVAL;
  }
  *stream = static_cast<void*>(s->st);
  return LAPH_OK;
}

int laph_solver_timings(laph_solver* s, double* ms4) {
  if (!s || !ms4) return LAPH_EINVAL;
  for (int i = 0; i < 4; ++i) ms4[i] = s->ms[i];
  return LAPH_OK;
}

int laph_solver_set_smear(laph_solver* s, int i, double p1, double p2) {
  if (!s || i < 0 || i >= s->np || !std::isfinite(p1) || !std::isfinite(p2)) {
    set_error("laph_solver_set_smear: bad argument");
    return LAPH_EINVAL;
  }
  if (s->sp1[i] != p1 || s->sp2[i] != p2) {
    s->sp1[i] = p1;
    s->sp2[i] = p2;
    if (s->g_solve) {  // its smearing launches carry the old parameters
      cudaGraphExecDestroy(s->g_solve);
      s->g_solve = nullptr;
    }
  }
  return LAPH_OK;
}

int laph_solver_sourceshape(laph_solver* s, int i, int weighted, double* psi) {
  if (!s || i < 0 || i >= s->np || !s->ran || !psi || (s->hd[i].L & 1)) {
    set_error("laph_solver_sourceshape: bad argument, solver not run, or odd L");
    return LAPH_EINVAL;
  }
  LAPH_CUDA_TRY(cudaSetDevice(s->dev));
  const ProbDesc& d = s->hd[i];
  const int H = d.L / 2, Nc = H * H * H;
  // scratch, both free once the run has finished and rewritten by the next run:
  // W (the class-major copy of the colour-major V), E0 (psi bins)
  double* dpsi = reinterpret_cast<double*>(s->E[0] + d.blk);
  LAPH_TRY(sourceshape_device(s->V + d.blk, d.L, d.nev, weighted ? s->theta + d.kv : nullptr, s->W + d.blk, dpsi, 1,
                              s->st));
  LAPH_CUDA_TRY(cudaMemcpyAsync(psi, dpsi, sizeof(double) * Nc, cudaMemcpyDeviceToHost, s->st));
  LAPH_CUDA_TRY(cudaStreamSynchronize(s->st));
  return LAPH_OK;
}

int laph_solver_displace(laph_solver* s, int i, int dir, double* W, int on_device) {
  if (!s || i < 0 || i >= s->np || !s->ran || !W || dir < 0 || dir > 2) {
    set_error("laph_solver_displace: bad argument or solver not run");
    return LAPH_EINVAL;
  }
  LAPH_CUDA_TRY(cudaSetDevice(s->dev));
  const ProbDesc& d = s->hd[i];
  // reads the colour-major V in place; host output goes through W, free after the run
  double2* out = on_device ? reinterpret_cast<double2*>(W) : s->W + d.blk;
  LAPH_TRY(displace_device(s->U64 + d.u64, d.L, dir, d.nev, d.dim, s->V + d.blk, out, 1, s->st));
  if (!on_device)
    LAPH_CUDA_TRY(cudaMemcpyAsync(W, out, sizeof(double2) * d.dim * d.nev, cudaMemcpyDeviceToHost, s->st));
  LAPH_CUDA_TRY(cudaStreamSynchronize(s->st));
  return LAPH_OK;
}

int laph_solver_loop_info(laph_solver* s, int* device_loop, long long* graph_launches) {
  if (!s || !device_loop || !graph_launches || !s->ran) {
    set_error("laph_solver_loop_info: bad argument or solver not run");
    return LAPH_EINVAL;
  }
  *device_loop = s->last_loop;
  *graph_launches = s->last_graph_launches;
  return LAPH_OK;
}

int laph_solver_filter_bytes(laph_solver* s, double* b2) {
  if (!s || !b2) {
    set_error("laph_solver_filter_bytes: bad argument");
    return LAPH_EINVAL;
  }
  b2[0] = s->fbytes[0];
  b2[1] = s->fbytes[1];
  return LAPH_OK;
}

int laph_solver_counters(laph_solver* s, long long* c3) {
  if (!s || !c3) return LAPH_EINVAL;
  for (int i = 0; i < 3; ++i) c3[i] = s->cnt[i];
  return LAPH_OK;
}

// Device bytes laph_solver_create allocates for probs[0..n): the same pool
// arithmetic as create (keep the two in step), every allocation rounded up to
// the 2 MiB the CUDA allocator hands out for large requests.  The CUDA graphs
// a run captures come on top (small: kernel nodes only).
int laph_solver_footprint(const laph_problem* probs, int n, const laph_solve_opts* opts, long long* bytes) {
  if (!probs || n < 1 || !opts || !bytes) {
    set_error("laph_solver_footprint: bad argument");
    return LAPH_EINVAL;
  }
  long long o_u64 = 0, o_uf = 0, o_sc = 0, o_blk = 0, o_kk = 0, o_kv = 0, o_gp = 0, o_rp = 0, o_tc = 0;
  long long max_run = 0, max_v3 = 0;
  for (int i = 0; i < n; ++i) {
    const long long L = probs[i].L, V3 = L * L * L, dim = 3 * V3;
    const int k = round_up(probs[i].nev + opts->guard, kGramTile);
    if (L < 3 || L > 128 || probs[i].nev < 1 || k > 512 || k > dim / 2) {
      set_error("laph_solver_footprint: problem %d is not solvable (see laph_solver_create)", i);
      return LAPH_EINVAL;
    }
    const long long nchunk = (dim + 8191) / 8192, T = k / kGramTile, npair = T * (T + 1) / 2;
    const long long mdeg = opts->deg > 0 ? opts->deg : 16;
    o_u64 += 27 * V3;
    o_uf += 27 * V3;
    o_sc += V3;
    o_blk += dim * k;
    o_kk += 5LL * k * k;
    o_kv += k;
    o_gp += nchunk * 2 * npair * kGramTile * kGramTile;
    o_rp += ((V3 + 127) / 128) * k;
    o_tc += (mdeg + 1) * 3 * k;
    max_v3 = std::max(max_v3, V3);
  }
  for (int i = 0; i < n;) {
    int j = i;
    while (j < n && probs[j].L == probs[i].L) ++j;
    max_run = std::max(max_run, (long long)(j - i) * 27 * probs[i].L * probs[i].L * probs[i].L);
    i = j;
  }
  const long long page = 2LL << 20;
  long long total = 0;
  auto add = [&](long long b) { total += (std::max(b, 1LL) + page - 1) / page * page; };
  add(n * (long long)sizeof(ProbDesc));
  add(n * (long long)sizeof(ProbState));
  add(o_u64 * 16);
  add(o_u64 * 16);
  add(max_run * 16);
  add(36 * max_v3 * 16);
  add(max_run * 2 * 16);
  add(o_sc * 4);
  for (int b = 0; b < 3; ++b) add(o_blk * 16);  // V, W, Y
  for (int b = 0; b < 4; ++b) add(o_blk * 8);   // S, E0..E2
  add(o_kk * 16);
  add(o_gp * 16);
  add(o_rp * 8);
  for (int b = 0; b < 4; ++b) add(o_kv * 8);  // theta, scol, resid, phases
  add(o_kv * 8);                              // norms
  add(o_tc * 8);
  add(4 * o_kv * 8);                          // dwork
  add(4);                                     // active count
  add((long long)(kMlpParams + kMlpNorm) * 4);
  add((long long)n * kMlpIn * 4);
  add((long long)n * (kMlpIn + kMlpOut) * 4);
  add((long long)n * 8);
  add(4LL * n * 8);
  add((long long)n * 4);
  add((long long)n * kSmallPhases * 8);
  add(o_uf * 8);                              // filter links (FP32, or BF16 + scale in the same pool)
  for (int t = 0; t < 9; ++t) add((n + 1) * 4LL);  // CTA -> problem prefix tables
  *bytes = total;
  return LAPH_OK;
}

int laph_solver_max_batch(const laph_problem* probs, int n, const laph_solve_opts* opts, int device, double fraction,
                          int* nmax) {
  if (!probs || n < 1 || !opts || !nmax || !(fraction > 0.0 && fraction <= 1.0)) {
    set_error("laph_solver_max_batch: bad argument");
    return LAPH_EINVAL;
  }
  long long need = 0;
  LAPH_TRY(laph_solver_footprint(probs, 1, opts, &need));  // validates the first problem before the device
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    set_error("laph_solver_max_batch: no CUDA device %d", device);
    return LAPH_ENODEV;
  }
  LAPH_CUDA_TRY(cudaSetDevice(device));
  size_t free_b = 0, total_b = 0;
  LAPH_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
  const double budget = fraction * (double)free_b;
  // largest m with footprint(probs[0..m)) within the budget (the footprint grows with m)
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    LAPH_TRY(laph_solver_footprint(probs, mid, opts, &need));
    if ((double)need <= budget) lo = mid;
    else hi = mid - 1;
  }
  *nmax = lo;
  if (lo == 0) {
    laph_solver_footprint(probs, 1, opts, &need);
    set_error("laph_solver_max_batch: one problem needs %lld bytes, %.0f of %zu free allowed", need, budget, free_b);
    return LAPH_ENOMEM;
  }
  return LAPH_OK;
}

}  // extern "C"
