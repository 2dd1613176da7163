// tune_hyp.cpp -- laph_tune_hyp, the replacement of LapH_EigSys's tune_hyp
// (src/tune_hyp.cpp): for one timeslice of a configuration, the lowest
// eigenpairs of -Delta after HYP smearing over a grid of (alpha_1, alpha_2),
// both stepping by 0.05 from alpha_*_i up to alpha_*_f with the reference's
// floating-point loop, ITER iterations each.  The reference smears and solves
// the grid points one after another; here every grid point is one problem of a
// batched device solve (a copy of the same links with its own smearing
// parameters, laph_solver_set_smear), in waves of as many grid points as fit
// in the device's free memory.  Outputs as the reference:
// <result_path>/eigenvalues_hyp-<iter>_a1-<a1>_a2-<a2>.<config>.<ts> and the
// phases_... files, then the table "#alpha1 alpha2 lowest_ev" on stdout.
// The reference hard-codes timeslice 10; --ts overrides it.
#include <algorithm>
#include <omp.h>

#include <cstdio>
#include <cstdlib>
#include <string>
#include <utility>
#include <vector>

#include "../../include/laph_gpu.h"
#include "cli_defaults.h"

namespace {

int die(int st, const char* what) {
  std::fprintf(stderr, "laph_tune_hyp: %s: %s (%s)\n", what, laph_strerror(st), laph_last_error());
  return 1;
}

// One grid point's two files, named as the reference names them, and its JSON line.
int write_point(const laph_config& P, int config, int ts, int nev, const std::pair<double, double>& a,
                const laph_result& r, const std::vector<double>& evals, const std::vector<double>& phases,
                double* lowest) {
  char ev_prefix[200], phs_prefix[200];
  std::snprintf(ev_prefix, sizeof ev_prefix, "eigenvalues_hyp-%d_a1-%.2f_a2-%.2f", P.iter, a.first, a.second);
  std::snprintf(phs_prefix, sizeof phs_prefix, "phases_hyp-%d_a1-%.2f_a2-%.2f", P.iter, a.first, a.second);
  int st = laph_write_eigenvalues_bin(P.result_path, ev_prefix, config, ts, nev, evals.data());
  if (st == LAPH_OK) st = laph_write_eigenvalues_bin(P.result_path, phs_prefix, config, ts, nev, phases.data());
  if (st != LAPH_OK) return st;
  *lowest = evals[0];
  std::printf("{\"alpha_1\": %.2f, \"alpha_2\": %.2f, \"status\": %d, \"iters\": %d, \"max_resid\": %.3e, "
              "\"lowest_ev\": %.12f}\n",
              a.first, a.second, r.status, r.iters, r.max_resid, evals[0]);
  return LAPH_OK;
}

}  // namespace

int main(int argc, char** argv) {
  int config = -1, ts = 10;
  std::string params = "parameters.txt";
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--ts" && i + 1 < argc) ts = std::atoi(argv[++i]);
    else if (a == "--parameters" && i + 1 < argc) params = argv[++i];
    else if (a == "--conf" && i + 1 < argc) config = std::atoi(argv[++i]);
    else if (i == argc - 1) config = std::atoi(argv[i]);  // the reference takes the config as the last argument
    else {
      std::fprintf(stderr, "usage: laph_tune_hyp [--ts T] [--parameters FILE] CONFIG\n");
      return 2;
    }
  }
  if (config < 0) {
    std::fprintf(stderr, "usage: laph_tune_hyp [--ts T] [--parameters FILE] CONFIG\n");
    return 2;
  }
  laph_config P;
  int st = laph_parse_parameters(params.c_str(), &P);
  if (st != LAPH_OK) return die(st, "parameters");
  // host threads (LIME reading, checks), as the reference's OMP_THRDS sets them (shell_matop.cpp:26)
  if (P.OMP_THRDS > 0) omp_set_num_threads(P.OMP_THRDS);
  const int L = P.LX, LT = P.LT, nev = P.NEV, V3 = L * L * L;
  if (ts < 0 || ts >= LT) {
    std::fprintf(stderr, "laph_tune_hyp: timeslice %d outside 0..%d\n", ts, LT - 1);
    return 2;
  }
  // the grid, with the reference's accumulation (for (a = a_i; a <= a_f; a += 0.05))
  std::vector<std::pair<double, double>> grid;
  for (double a1 = P.alpha_1_i; a1 <= P.alpha_1_f; a1 += 0.05)
    for (double a2 = P.alpha_2_i; a2 <= P.alpha_2_f; a2 += 0.05) grid.emplace_back(a1, a2);
  if (grid.empty()) {
    std::fprintf(stderr, "laph_tune_hyp: empty (alpha_1, alpha_2) grid\n");
    return 2;
  }
  char conf_name[1100];
  std::snprintf(conf_name, sizeof conf_name, "%s/conf.%04d", P.config_path, config);
  std::vector<double> conf((size_t)V3 * 72);
  int prec = 64;
  st = laph_lime_read_gauge_any(conf_name, LT, L, ts, ts, conf.data(), &prec);
  if (st != LAPH_OK) return die(st, "read gauge");
  const int n = (int)grid.size();
  std::vector<laph_problem> probs(n, laph_problem{L, nev});
  laph_solve_opts o;
  laph_solve_opts_default(&o);
  o.smear_kind = LAPH_SMEAR_HYP;
  o.smear_iters = P.iter;
  o.smear_compat = 1;
  o.guard = P.guard;
  o.tol = P.tol > 0 ? P.tol : 1e-9;
  o.block = P.block;
  o.deg = P.filter_deg > 0 ? P.filter_deg : default_filter_deg(L, o.deg);
  const int device = std::getenv("LAPH_DEVICE") ? std::atoi(std::getenv("LAPH_DEVICE")) : 0;
  // waves of as many grid points as one solver fits in the device's free memory
  int wave = n;
  st = laph_solver_max_batch(probs.data(), n, &o, device, 0.85, &wave);
  if (st != LAPH_OK) return die(st, "device memory");
  laph_solver* s = nullptr;
  int s_np = 0;
  std::vector<laph_result> res(n);
  std::vector<double> evals(nev), phases(nev), lowest(n);
  for (int w0 = 0; w0 < n; w0 += wave) {
    const int wn = std::min(wave, n - w0);
    if (wn != s_np) {
      laph_solver_destroy(s);
      s = nullptr;
      st = laph_solver_create(&s, probs.data() + w0, wn, &o, device);
      if (st != LAPH_OK) return die(st, "solver");
      s_np = wn;
    }
    for (int i = 0; i < wn; ++i) {
      st = laph_solver_set_links(s, i, conf.data(), LAPH_LAYOUT_CONF, 0);
      if (st == LAPH_OK) st = laph_solver_set_smear(s, i, grid[w0 + i].first, grid[w0 + i].second);
      if (st != LAPH_OK) return die(st, "links");
    }
    st = laph_solver_run(s, res.data() + w0);
    if (st != LAPH_OK && st != LAPH_ENOTCONV) return die(st, "solve");
    for (int i = 0; i < wn; ++i) {
      st = laph_solver_get(s, i, evals.data(), nullptr, phases.data(), 0);
      if (st != LAPH_OK) return die(st, "fetch");
      st = write_point(P, config, ts, nev, grid[w0 + i], res[w0 + i], evals, phases, &lowest[w0 + i]);
      if (st != LAPH_OK) return die(st, "write");
    }
  }
  laph_solver_destroy(s);
  std::printf("#alpha1\talpha2\tlowest_ev\n");
  for (int i = 0; i < n; ++i) std::printf("%g\t%g\t%.12g\n", grid[i].first, grid[i].second, lowest[i]);
  return 0;
}
