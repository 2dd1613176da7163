// autotune.cpp -- the block solver's autotuner.  Three settings trade filter
// work against outer iterations and kernel efficiency, and their best values
// move with the lattice, nev, the link precision and the part's clock:
//
//   deg    the filter degree cap (more damping per pass, fewer Rayleigh-Ritz)
//   block  columns per CTA of the filter kernel (links read once per block)
//   guard  vectors beyond nev, hence the block width k (faster convergence of
//          the wanted pairs against more work per pass)
//   tile   sites per CTA of the filter (64, 128, 256: the shared-memory share
//          of the backward links and the prefetch run per CTA), tried last
//          with the other three at their best
//
// laph_autotune_search walks them one axis at a time (deg, then block, then
// guard; each candidate of an axis timed with the others at their best so far,
// a candidate kept only when it is more than 1% faster), every setting timed
// at most once.  laph_solver_autotune times each setting as a real solve of a
// sample of the batch (the faster of two runs of one solver: the first also
// captures the CUDA graphs) and keeps the result in an optional cache file,
// one line per device and batch shape, so a production run tunes once.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/laph_gpu.h"

namespace laph {
void set_error(const char* fmt, ...);
}
using laph::set_error;

namespace {

constexpr double kTuneMargin = 0.01;  // a candidate must be this much faster to replace the best

struct SampleCtx {
  const laph_problem* probs;
  int ns;
  const double* const* links;
  int layout;
  laph_solve_opts base;
  const float* model;
  int nmodel;
  int device;
  int last_status;
  int tile;  // filter sites per CTA of the trials
};

// One setting: device milliseconds per problem of the faster of two runs, or -1.
double sample_trial(void* user, int deg, int block, int guard) {
  SampleCtx* c = static_cast<SampleCtx*>(user);
  laph_solve_opts o = c->base;
  o.deg = deg;
  o.block = block;
  o.guard = guard;
  o.filter_tile = c->tile;
  laph_solver* s = nullptr;
  int st = laph_solver_create(&s, c->probs, c->ns, &o, c->device);
  c->last_status = st;
  if (st != LAPH_OK) return -1.0;
  double best = -1.0;
  if (o.window == LAPH_WINDOW_MLP) st = laph_solver_set_window_model(s, c->model, c->nmodel);
  for (int i = 0; i < c->ns && st == LAPH_OK; ++i) st = laph_solver_set_links(s, i, c->links[i], c->layout, 0);
  for (int rep = 0; rep < 2 && st == LAPH_OK; ++rep) {
    st = laph_solver_run(s, nullptr);
    double ms[4] = {0, 0, 0, 0};
    if (st == LAPH_OK && laph_solver_timings(s, ms) == LAPH_OK && ms[3] > 0.0) {
      const double per = ms[3] / c->ns;
      best = best < 0.0 ? per : std::min(best, per);
    }
  }
  c->last_status = st;
  laph_solver_destroy(s);
  return st == LAPH_OK ? best : -1.0;
}

std::string shape_key(const cudaDeviceProp& prop, const laph_problem* probs, int ns, const laph_solve_opts* o) {
  std::string k = prop.name;
  char buf[256];
  std::snprintf(buf, sizeof buf, "|sm_%d%d|", prop.major, prop.minor);
  k += buf;
  for (int i = 0; i < ns; ++i) {
    std::snprintf(buf, sizeof buf, "%sL%dn%d", i ? "," : "", probs[i].L, probs[i].nev);
    k += buf;
  }
  std::snprintf(buf, sizeof buf, "|prec%d|smear%d:%.6g:%.6g:%d:%d|tol%.3g|win%d|fk%d|g%d|it%d", o->link_prec,
                o->smear_kind, o->smear_p1, o->smear_p2, o->smear_iters, o->smear_compat, o->tol, o->window,
                o->filter_kernel, o->guard, o->max_it);
  k += buf;
  for (char& ch : k)
    if (ch == '\t' || ch == '\n') ch = ' ';
  return k;
}

// "key<TAB>deg block guard ms [tile]" lines; the last line with the key wins.
bool cache_lookup(const char* path, const std::string& key, laph_tune_result* r) {
  FILE* f = std::fopen(path, "r");
  if (!f) return false;
  bool found = false;
  std::vector<char> line(8192);
  while (std::fgets(line.data(), (int)line.size(), f)) {
    const char* tab = std::strchr(line.data(), '\t');
    if (!tab || std::string(line.data(), (size_t)(tab - line.data())) != key) continue;
    int d = 0, b = 0, g = 0, t = 0;
    double ms = 0.0;
    const int n = std::sscanf(tab + 1, "%d %d %d %lf %d", &d, &b, &g, &ms, &t);
    if (n >= 4) {
      r->deg = d;
      r->block = b;
      r->guard = g;
      r->ms_per_problem = ms;
      r->tile = n == 5 ? t : 128;
      found = true;
    }
  }
  std::fclose(f);
  return found;
}

}  // namespace

extern "C" {

int laph_autotune_search(const int* deg_c, int nd, const int* block_c, int nb, const int* guard_c, int ng, int deg0,
                         int block0, int guard0, laph_tune_trial trial, void* user, laph_tune_result* out) {
  if (!trial || !out || nd < 0 || nb < 0 || ng < 0 || (nd && !deg_c) || (nb && !block_c) || (ng && !guard_c)) {
    set_error("laph_autotune_search: bad argument");
    return LAPH_EINVAL;
  }
  std::map<std::tuple<int, int, int>, double> memo;
  auto eval = [&](int d, int b, int g) {
    const auto key = std::make_tuple(d, b, g);
    auto it = memo.find(key);
    if (it != memo.end()) return it->second;
    double ms = trial(user, d, b, g);
    if (!(ms >= 0.0) || !std::isfinite(ms)) ms = INFINITY;
    memo[key] = ms;
    return ms;
  };
  int cur[3] = {deg0, block0, guard0};
  double best = eval(cur[0], cur[1], cur[2]);
  const int* cand[3] = {deg_c, block_c, guard_c};
  const int count[3] = {nd, nb, ng};
  for (int axis = 0; axis < 3; ++axis) {
    int keep = cur[axis];
    for (int i = 0; i < count[axis]; ++i) {
      int p[3] = {cur[0], cur[1], cur[2]};
      p[axis] = cand[axis][i];
      const double ms = eval(p[0], p[1], p[2]);
      if (ms < best * (1.0 - kTuneMargin) || (!std::isfinite(best) && std::isfinite(ms))) {
        best = ms;
        keep = p[axis];
      }
    }
    cur[axis] = keep;
  }
  out->trials = (int)memo.size();
  out->from_cache = 0;
  if (!std::isfinite(best)) {
    set_error("laph_autotune_search: none of the %d settings tried succeeded", out->trials);
    return LAPH_ENOTCONV;
  }
  out->deg = cur[0];
  out->block = cur[1];
  out->guard = cur[2];
  out->ms_per_problem = best;
  return LAPH_OK;
}

int laph_solver_autotune(const laph_problem* probs, int n, const double* const* links, int layout, int nsample,
                         laph_solve_opts* opts, const float* model, int nmodel, int device, const char* cache_path,
                         laph_tune_result* out) {
  if (!probs || n < 1 || !links || nsample < 1 || !opts || !out) {
    set_error("laph_solver_autotune: bad argument");
    return LAPH_EINVAL;
  }
  if (opts->window == LAPH_WINDOW_MLP && (!model || nmodel < 1)) {
    set_error("laph_solver_autotune: window = MLP needs the window model");
    return LAPH_EINVAL;
  }
  const int ns = std::min(n, nsample);
  for (int i = 0; i < ns; ++i)
    if (!links[i]) {
      set_error("laph_solver_autotune: links of sample problem %d missing", i);
      return LAPH_EINVAL;
    }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    set_error("laph_solver_autotune: no CUDA device %d", device);
    return LAPH_ENODEV;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
    cudaGetLastError();
    set_error("laph_solver_autotune: cannot query device %d", device);
    return LAPH_ENODEV;
  }
  const std::string key = shape_key(prop, probs, ns, opts);
  std::memset(out, 0, sizeof *out);
  if (cache_path && *cache_path && cache_lookup(cache_path, key, out)) {
    out->from_cache = 1;
    opts->deg = out->deg;
    opts->block = out->block;
    opts->guard = out->guard;
    opts->filter_tile = out->tile;
    return LAPH_OK;
  }
  const int deg0 = opts->deg > 1 ? std::min(opts->deg, 96) : 60;
  const int block0 = opts->block > 0 ? opts->block : 32;
  const int guard0 = opts->guard;
  const int degs[] = {40, 48, 56, 60, 64, 72, 80, 96};
  const int blocks[] = {8, 16, 32, 64};
  // guard: the given one, 32 more, and the fewest (>= 4) that keep the block width at its smallest multiple of 32
  // (nev 120: guard 8, k = 128 instead of 160 -- less work per pass against slower convergence of the top pairs)
  const int gmin = std::max(4, ((probs[0].nev + 4 + 31) / 32) * 32 - probs[0].nev);
  std::vector<int> guards = {guard0, guard0 + 32};
  if (gmin != guard0 && gmin != guard0 + 32 && ((probs[0].nev + gmin + 31) / 32 != (probs[0].nev + guard0 + 31) / 32))
    guards.push_back(gmin);
  const int tile0 = opts->filter_tile > 0 ? opts->filter_tile : 128;
  SampleCtx ctx{probs, ns, links, layout, *opts, model, nmodel, device, LAPH_OK, tile0};
  int st = laph_autotune_search(degs, 8, blocks, 4, guards.data(), (int)guards.size(), deg0, block0, guard0,
                                sample_trial, &ctx, out);
  if (st != LAPH_OK) {
    if (ctx.last_status != LAPH_OK && ctx.last_status != LAPH_ENOTCONV)
      set_error("laph_solver_autotune: every setting failed; the last with status %d (%s)", ctx.last_status,
                laph_strerror(ctx.last_status));
    return st;
  }
  // the tile axis, with deg / block / guard at their best (the kernel variant
  // with FP32 coefficients per CTA only: wider blocks keep 128 sites)
  out->tile = tile0;
  if (opts->filter_kernel == 1 && out->block <= 64) {
    for (int t : {64, 128, 256}) {
      if (t == tile0) continue;
      ctx.tile = t;
      const double ms = sample_trial(&ctx, out->deg, out->block, out->guard);
      ++out->trials;
      if (ms > 0.0 && ms < (1.0 - kTuneMargin) * out->ms_per_problem) {
        out->ms_per_problem = ms;
        out->tile = t;
      }
    }
  }
  opts->deg = out->deg;
  opts->block = out->block;
  opts->guard = out->guard;
  opts->filter_tile = out->tile;
  if (cache_path && *cache_path) {
    FILE* f = std::fopen(cache_path, "a");
    if (!f) {
      set_error("laph_solver_autotune: cannot append to %s", cache_path);
      return LAPH_EIO;
    }
    std::fprintf(f, "%s\t%d %d %d %.6f %d\n", key.c_str(), out->deg, out->block, out->guard, out->ms_per_problem,
                 out->tile);
    std::fclose(f);
  }
  return LAPH_OK;
}

}  // extern "C"
