// integration_examples.cpp -- the C++ code of the integration guide, as it
// goes into the reference's programs (src/ev_ts.cpp, src/tune_hyp.cpp), each
// block inside a function that declares the variables the reference has in
// scope at that point.  tests/test_integration_snippets.py compiles this file
// against the shipped headers (include/laph_matshell.h over
// include/petsc_shim.h), so the examples cannot drift from the ABI.  Not
// linked into anything.

#include <cstdio>
#include <vector>
#include "../../include/laph_matshell.h"
struct ref_io { double get_float(const char*); int get_int(const char*); };  // the reference's IO singleton

// ---- guide block 1
int example_1() {

  ref_io* pars = nullptr; (void)pars;
  int L1 = 24, todo = 4, nev = 120, ITER = 3, config = 1227, tstart = 0, MAT_ENTRIES = 3 * 24 * 24 * 24;
  int V_TS = 72 * 24 * 24 * 24, ngrid = 4, ts = 0;
  double ALPHA_1 = 0.62, ALPHA_2 = 0.52;
  double* configuration = nullptr; double* timeslice = nullptr; double* evals = nullptr;
  double alpha1[4] = {0}, alpha2[4] = {0};
  std::vector<double> eigensystem_fix, phase;
  laph_result* results = nullptr;
  const char* result_path = ".";
  PetscErrorCode ierr = 0; Mat A = nullptr; (void)ierr; (void)A;
  (void)L1; (void)todo; (void)nev; (void)ITER; (void)config; (void)tstart; (void)MAT_ENTRIES; (void)V_TS;
  (void)ngrid; (void)ts; (void)ALPHA_1; (void)ALPHA_2; (void)configuration; (void)timeslice; (void)evals;
  (void)alpha1; (void)alpha2; (void)results; (void)result_path;

  laph_solver* s = nullptr;
// (real PETSc in the guide; the shim here)          // build against the real PETSc/SLEPc

// once, before the timeslice loop (replaces Nav::init / Tslice::init)
laph_params lp = {L1, pars->get_float("lambda_l"), pars->get_float("lambda_c"), pars->get_int("DEG"), /*device*/ 0};
laph_ctx* gpu = nullptr;
if (laph_ctx_create(&gpu, &lp) != LAPH_OK) { fprintf(stderr, "%s\n", laph_last_error()); return 1; }
laph_shell shell = {gpu, pars->get_int("DEG")};

for (int ts = 0; ts < todo; ++ts) {
  double* timeslice = configuration + ts * V_TS;
  laph_set_links(gpu, timeslice, LAPH_LAYOUT_CONF);             // map_timeslice_to_eigen
  laph_smear(gpu, LAPH_SMEAR_HYP, ALPHA_1, ALPHA_2, ITER, 0);   // slice->smearing_hyp(...)
  ierr = MatCreateShell(PETSC_COMM_SELF, PETSC_DECIDE, PETSC_DECIDE, MAT_ENTRIES, MAT_ENTRIES, &shell, &A);
  ierr = MatShellSetOperation(A, MATOP_MULT, (void(*)())MatMult_Laplacian2D_GPU);
  ierr = MatShellSetOperation(A, MATOP_MULT_TRANSPOSE, (void(*)())MatMult_Laplacian2D_GPU);
  ierr = MatShellSetOperation(A, MATOP_GET_DIAGONAL, (void(*)())MatGetDiagonal_Laplacian2D_GPU);
  /* ... EPSCreate / EPSSolve / EPSGetEigenpair / fix_phase / recover_spectrum unchanged ... */
}
laph_ctx_destroy(gpu);
  return 0;
}

// ---- guide block 2
int example_2() {

  ref_io* pars = nullptr; (void)pars;
  int L1 = 24, todo = 4, nev = 120, ITER = 3, config = 1227, tstart = 0, MAT_ENTRIES = 3 * 24 * 24 * 24;
  int V_TS = 72 * 24 * 24 * 24, ngrid = 4, ts = 0;
  double ALPHA_1 = 0.62, ALPHA_2 = 0.52;
  double* configuration = nullptr; double* timeslice = nullptr; double* evals = nullptr;
  double alpha1[4] = {0}, alpha2[4] = {0};
  std::vector<double> eigensystem_fix, phase;
  laph_result* results = nullptr;
  const char* result_path = ".";
  PetscErrorCode ierr = 0; Mat A = nullptr; (void)ierr; (void)A;
  (void)L1; (void)todo; (void)nev; (void)ITER; (void)config; (void)tstart; (void)MAT_ENTRIES; (void)V_TS;
  (void)ngrid; (void)ts; (void)ALPHA_1; (void)ALPHA_2; (void)configuration; (void)timeslice; (void)evals;
  (void)alpha1; (void)alpha2; (void)results; (void)result_path;

std::vector<laph_problem> probs(todo, laph_problem{L1, nev});
laph_solve_opts o; laph_solve_opts_default(&o);
o.smear_kind = LAPH_SMEAR_HYP; o.smear_p1 = ALPHA_1; o.smear_p2 = ALPHA_2; o.smear_iters = ITER;
o.tol = 1e-9;                       // ||(-Delta) v - lambda v|| / (||v|| * 12)
o.window = LAPH_WINDOW_MLP;         // learned first window (data/window_mlp.bin via laph_solver_set_window_model)
o.deg = 60;                         // filter degree cap (60 measured best at 24^3-32^3; laph_solver_autotune picks it)
laph_solver* s; laph_solver_create(&s, probs.data(), todo, &o, /*device*/ 0);
for (int ts = 0; ts < todo; ++ts) laph_solver_set_links(s, ts, configuration + ts * V_TS, LAPH_LAYOUT_CONF, 0);
laph_solver_run(s, results);        // LAPH_ENOTCONV if a timeslice did not converge (the reference ignores this)
for (int ts = 0; ts < todo; ++ts) {
  laph_solver_get(s, ts, evals, eigensystem_fix.data(), phase.data(), 0);   // phase-fixed, column-major
  laph_write_eigsys_bin(result_path, "eigenvectors", config, tstart + ts, MAT_ENTRIES, nev, eigensystem_fix.data());
  laph_write_eigenvalues_bin(result_path, "eigenvalues", config, tstart + ts, nev, evals);
  laph_write_eigenvalues_bin(result_path, "phases", config, tstart + ts, nev, phase.data());
}
laph_solver_destroy(s);
  return 0;
}

// ---- guide block 3
int example_3() {

  ref_io* pars = nullptr; (void)pars;
  int L1 = 24, todo = 4, nev = 120, ITER = 3, config = 1227, tstart = 0, MAT_ENTRIES = 3 * 24 * 24 * 24;
  int V_TS = 72 * 24 * 24 * 24, ngrid = 4, ts = 0;
  double ALPHA_1 = 0.62, ALPHA_2 = 0.52;
  double* configuration = nullptr; double* timeslice = nullptr; double* evals = nullptr;
  double alpha1[4] = {0}, alpha2[4] = {0};
  std::vector<double> eigensystem_fix, phase;
  laph_result* results = nullptr;
  const char* result_path = ".";
  PetscErrorCode ierr = 0; Mat A = nullptr; (void)ierr; (void)A;
  (void)L1; (void)todo; (void)nev; (void)ITER; (void)config; (void)tstart; (void)MAT_ENTRIES; (void)V_TS;
  (void)ngrid; (void)ts; (void)ALPHA_1; (void)ALPHA_2; (void)configuration; (void)timeslice; (void)evals;
  (void)alpha1; (void)alpha2; (void)results; (void)result_path;

std::vector<laph_problem> probs(todo, laph_problem{L1, nev});
laph_solve_opts o; laph_solve_opts_default(&o);
std::vector<float> model;           // data/window_mlp.bin when o.window = LAPH_WINDOW_MLP
std::vector<const double*> sample;  // links of the first timeslices
for (int ts = 0; ts < 4 && ts < todo; ++ts) sample.push_back(configuration + ts * V_TS);
laph_tune_result tr;
laph_solver_autotune(probs.data(), todo, sample.data(), LAPH_LAYOUT_CONF, (int)sample.size(), &o,
                     model.empty() ? nullptr : model.data(), (int)model.size(), /*device*/ 0, "tune.txt", &tr);
int wave = todo;
laph_solver_max_batch(probs.data(), todo, &o, /*device*/ 0, 0.85, &wave);  // timeslices per solver
  return 0;
}

// ---- guide block 4
int example_4() {

  ref_io* pars = nullptr; (void)pars;
  int L1 = 24, todo = 4, nev = 120, ITER = 3, config = 1227, tstart = 0, MAT_ENTRIES = 3 * 24 * 24 * 24;
  int V_TS = 72 * 24 * 24 * 24, ngrid = 4, ts = 0;
  double ALPHA_1 = 0.62, ALPHA_2 = 0.52;
  double* configuration = nullptr; double* timeslice = nullptr; double* evals = nullptr;
  double alpha1[4] = {0}, alpha2[4] = {0};
  std::vector<double> eigensystem_fix, phase;
  laph_result* results = nullptr;
  const char* result_path = ".";
  PetscErrorCode ierr = 0; Mat A = nullptr; (void)ierr; (void)A;
  (void)L1; (void)todo; (void)nev; (void)ITER; (void)config; (void)tstart; (void)MAT_ENTRIES; (void)V_TS;
  (void)ngrid; (void)ts; (void)ALPHA_1; (void)ALPHA_2; (void)configuration; (void)timeslice; (void)evals;
  (void)alpha1; (void)alpha2; (void)results; (void)result_path;

  laph_solver* s = nullptr;
std::vector<double> psi((L1 / 2) * (L1 / 2) * (L1 / 2)), r(psi.size()), avg(psi.size());
int n = 0;
laph_solver_sourceshape(s, ts, /*weighted*/ 0, psi.data());       // source_shape_complete
laph_sourceshape_avg(L1, psi.data(), r.data(), avg.data(), &n);   // avg_radii
laph_write_sourceshape(nullptr, config, tstart + ts, nev, n, r.data(), avg.data());  // write_sourceshape_ascii/_bin
  return 0;
}

// ---- guide block 5
int example_5() {

  ref_io* pars = nullptr; (void)pars;
  int L1 = 24, todo = 4, nev = 120, ITER = 3, config = 1227, tstart = 0, MAT_ENTRIES = 3 * 24 * 24 * 24;
  int V_TS = 72 * 24 * 24 * 24, ngrid = 4, ts = 0;
  double ALPHA_1 = 0.62, ALPHA_2 = 0.52;
  double* configuration = nullptr; double* timeslice = nullptr; double* evals = nullptr;
  double alpha1[4] = {0}, alpha2[4] = {0};
  std::vector<double> eigensystem_fix, phase;
  laph_result* results = nullptr;
  const char* result_path = ".";
  PetscErrorCode ierr = 0; Mat A = nullptr; (void)ierr; (void)A;
  (void)L1; (void)todo; (void)nev; (void)ITER; (void)config; (void)tstart; (void)MAT_ENTRIES; (void)V_TS;
  (void)ngrid; (void)ts; (void)ALPHA_1; (void)ALPHA_2; (void)configuration; (void)timeslice; (void)evals;
  (void)alpha1; (void)alpha2; (void)results; (void)result_path;

  laph_solver* s = nullptr;
for (int i = 0; i < ngrid; ++i) {
  laph_solver_set_links(s, i, timeslice, LAPH_LAYOUT_CONF, 0);
  laph_solver_set_smear(s, i, alpha1[i], alpha2[i]);   // kind and iterations from laph_solve_opts
}
laph_solver_run(s, results);
  return 0;
}

// ---- guide block: streaming several configurations with overlapped read-back
int example_streaming(laph_solver* s, laph_result* results, double* const* configs, int nconf, int todo, int V_TS,
                      double* const* const* ev_buf, double* const* const* vec_buf, double* const* const* ph_buf) {
  for (int c = 0; c < nconf; ++c) {
    for (int ts = 0; ts < todo; ++ts) laph_solver_set_links(s, ts, configs[c] + ts * V_TS, LAPH_LAYOUT_CONF, 0);
    laph_solver_run(s, results);
    for (int ts = 0; ts < todo; ++ts)   // buffers of configuration c, page-locked (cudaHostAlloc)
      laph_solver_get_async(s, ts, ev_buf[c][ts], vec_buf[c][ts], ph_buf[c][ts]);
  }
  laph_solver_wait(s);                  // every queued copy has landed
  return 0;
}
