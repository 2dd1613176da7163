// ev_ts.cpp -- laph_ev_ts, the command-line replacement for LapH_EigSys's
// ev_ts (src/ev_ts.cpp): same flags (--conf N, --phase_reset), same
// parameters.txt in the working directory, same input (<config_path>/conf.%04d
// LIME/ILDG) and outputs (<result_path>/eigenvectors|eigenvalues|phases.%04d.%03d).
//
//   solver = plain (parameters.txt): the reference's loop body -- link map,
//            smearing, MatShell with the GPU MatMult, EPS Krylov-Schur on
//            T_DEG(B), fix_phase, recover_spectrum -- one timeslice at a time.
//   solver = block (default): all timeslices of this process in batched
//            device solves (laph_solver), in waves of as many timeslices as
//            fit in the device's free memory (laph_solver_max_batch), same
//            outputs.
// Timeslices are split across processes as the reference splits them across
// MPI ranks (src/ev_ts.cpp:103-119): with the rank and size of the launcher
// (LAPH_RANK / LAPH_WORLD_SIZE, torchrun, mpirun, srun) rank r gets a
// contiguous block, the first LT % size ranks one extra.  One JSON line per timeslice goes to stdout.
// Beyond the reference: FP32 ILDG input is read (widened to FP64), and
// --resume skips timeslices whose three output files are already complete
// (right sizes, eigenvectors passing check_trace).
#include <omp.h>
#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <string>
#include <vector>

#include "../../include/laph_gpu.h"
#include "../../include/laph_matshell.h"
#include "cli_defaults.h"

namespace {

void usage() {
  std::fprintf(stderr,
               "usage: laph_ev_ts --conf N [--phase_reset 0|1] [--parameters FILE] [--resume]\n"
               "  reads parameters.txt (keys of LapH_EigSys plus smear, rho, alpha, tol, guard, block, filter_deg,\n"
               "  window, solver, autotune)\n");
}

// The first of the named environment variables that is set, as an int.
int env_int(std::initializer_list<const char*> names, int def) {
  for (const char* n : names)
    if (const char* v = std::getenv(n)) return std::atoi(v);
  return def;
}

// Rank, size and node-local rank of this process, all three taken from ONE
// launcher's variables: this program's own (LAPH_RANK / LAPH_WORLD_SIZE /
// LAPH_DEVICE), torchrun's, Open MPI's, MPICH / Intel MPI's (PMI) or Slurm's,
// the first launcher whose rank and size are both set.  Slurm counts only
// inside an srun step (SLURM_STEP_ID set; size SLURM_STEP_NUM_TASKS): a plain
// process in an sbatch allocation also sees SLURM_NTASKS / SLURM_PROCID, which
// describe the allocation, not this run.  Without a launcher: rank 0 of 1.
struct Launch {
  const char* name;
  int rank, size, local;
};
Launch launcher() {
  struct Vars {
    const char *name, *rank, *size, *local, *needs;
  };
  static const Vars kLaunchers[] = {
      {"laph", "LAPH_RANK", "LAPH_WORLD_SIZE", "LAPH_DEVICE", nullptr},
      {"torchrun", "RANK", "WORLD_SIZE", "LOCAL_RANK", nullptr},
      {"openmpi", "OMPI_COMM_WORLD_RANK", "OMPI_COMM_WORLD_SIZE", "OMPI_COMM_WORLD_LOCAL_RANK", nullptr},
      {"pmi", "PMI_RANK", "PMI_SIZE", "MPI_LOCALRANKID", nullptr},
      {"srun", "SLURM_PROCID", "SLURM_STEP_NUM_TASKS", "SLURM_LOCALID", "SLURM_STEP_ID"},
  };
  for (const Vars& v : kLaunchers) {
    if (!std::getenv(v.rank) || !std::getenv(v.size) || (v.needs && !std::getenv(v.needs))) continue;
    // LAPH_DEVICE picks the GPU under any launcher
    return Launch{v.name, env_int({v.rank}, 0), env_int({v.size}, 1), env_int({"LAPH_DEVICE", v.local}, 0)};
  }
  return Launch{"none", 0, 1, env_int({"LAPH_DEVICE"}, 0)};
}

int die(int st, const char* what) {
  std::fprintf(stderr, "laph_ev_ts: %s: %s (%s)\n", what, laph_strerror(st), laph_last_error());
  return 1;
}

// The learned-window model shipped next to the executable (data/window_mlp.bin):
// "LAPHMLP1", int32 nparams, int32 nnorm, float32[nparams + nnorm].
bool load_window_model(const char* exe, std::vector<float>* model) {
  std::string dir(exe);
  const size_t slash = dir.find_last_of('/');
  dir = slash == std::string::npos ? std::string(".") : dir.substr(0, slash);
  FILE* f = std::fopen((dir + "/data/window_mlp.bin").c_str(), "rb");
  if (!f) return false;
  char magic[8];
  int sizes[2];
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "LAPHMLP1", 8) == 0 &&
            std::fread(sizes, sizeof(int), 2, f) == 2 && sizes[0] == laph_mlp_nparams();
  if (ok) {
    model->resize(sizes[0] + sizes[1]);
    ok = std::fread(model->data(), sizeof(float), model->size(), f) == model->size();
  }
  std::fclose(f);
  return ok;
}

// A timeslice's outputs are complete when all three files have their full
// size and the eigenvectors pass check_trace (what the writer checks first).
bool outputs_complete(const char* dir, int config, int t, int dim, int nev) {
  static const char* kinds[3] = {"eigenvectors", "eigenvalues", "phases"};
  for (int k = 0; k < 3; ++k) {
    char name[1200];
    std::snprintf(name, sizeof name, "%s/%s.%04d.%03d", dir, kinds[k], config, t);
    struct stat sb;
    const long long want = k == 0 ? 16LL * dim * nev : 8LL * nev;
    if (stat(name, &sb) != 0 || (long long)sb.st_size != want) return false;
  }
  std::vector<double> V((size_t)2 * dim * nev);
  if (laph_read_eigsys_bin(dir, "eigenvectors", config, t, dim, nev, V.data()) != LAPH_OK) return false;
  double tr = 0.0, sum = 0.0;
  return laph_check_trace(dim, nev, V.data(), &tr, &sum) == 1;
}

// The run's settings on stdout before any work, as the reference's rank 0
// prints them (IO::print_summary, modules/par_io.cpp:138-154), plus this
// program's own keys; every line starts with '#' so that the JSON lines that
// follow stay easy to pick out.
void print_summary(const laph_config& P) {
  const long long V3 = (long long)P.LX * P.LX * P.LX;
  static const char* smear[] = {"none", "hyp", "stout", "ape"};
  static const char* window[] = {"fixed", "lanczos", "mlp"};
  std::printf("# lattice %d x %d x %d x %d, nev %d\n", P.LT, P.LX, P.LX, P.LX, P.NEV);
  std::printf("# smearing %s: alpha_1 %g alpha_2 %g rho %g alpha %g, %d iterations\n",
              smear[P.smear >= 0 && P.smear < 4 ? P.smear : 0], P.alpha_1, P.alpha_2, P.rho, P.alpha, P.iter);
  std::printf("# Chebyshev (plain form): LAM_L %g LAM_C %g DEG %d\n", P.LAM_L, P.LAM_C, P.DEG);
  std::printf("# solver %s, tol %g, guard %d, window %s, filter_deg %d, autotune %d\n", P.solver ? "plain" : "block",
              P.tol, P.guard, window[P.window >= 0 && P.window < 3 ? P.window : 1], P.filter_deg, P.autotune);
  std::printf("# configurations from %s, results to %s\n", P.config_path, P.result_path);
  std::printf("# MAT_ENTRIES %lld, V3 %lld, doubles per configuration %lld, OMP_THRDS %d\n", 3 * V3, V3,
              72 * V3 * P.LT, P.OMP_THRDS);
}

double trace_vdv(int dim, int nev, const double* V) {
  double tr = 0.0, sum = 0.0;
  laph_check_trace(dim, nev, V, &tr, &sum);
  return tr;
}

}  // namespace

int main(int argc, char** argv) {
  int config = -1, phase_reset = 0, resume = 0;
  std::string params = "parameters.txt";
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if ((a == "--conf") && i + 1 < argc) config = std::atoi(argv[++i]);
    else if (a.rfind("--conf=", 0) == 0) config = std::atoi(a.c_str() + 7);
    else if (a == "--phase_reset" && i + 1 < argc) phase_reset = std::atoi(argv[++i]);
    else if (a == "--parameters" && i + 1 < argc) params = argv[++i];
    else if (a == "--resume") resume = 1;
    else if (a == "--help") {
      usage();
      return 1;
    } else {
      usage();
      return 2;
    }
  }
  if (config < 0) {
    std::printf("No configuration number specified!\n");
    usage();
    return 2;
  }
  std::printf("Working on configuration %d\n", config);
  laph_config P;
  int st = laph_parse_parameters(params.c_str(), &P);
  if (st != LAPH_OK) return die(st, "parameters");
  // host threads (LIME reading, checks), as the reference's OMP_THRDS sets them (shell_matop.cpp:26)
  if (P.OMP_THRDS > 0) omp_set_num_threads(P.OMP_THRDS);
  const int L = P.LX, LT = P.LT, nev = P.NEV;
  const int V3 = L * L * L, dim = 3 * V3;
  const Launch ln = launcher();
  const int size = ln.size, rank = ln.rank, device = ln.local;
  if (rank == 0) {
    print_summary(P);
    std::printf("calculating config %d\n", config);
  }
  int t0, ntodo;
  st = laph_timeslice_split(LT, size, rank, &t0, &ntodo);
  if (st != LAPH_OK) return die(st, "timeslice split");
  // every rank says which part it took, so a wrong launcher guess shows at once
  std::printf("{\"launcher\": \"%s\", \"rank\": %d, \"size\": %d, \"device\": %d, \"t0\": %d, \"t1\": %d}\n", ln.name,
              rank, size, device, t0, t0 + ntodo - 1);
  char conf_name[1100];
  std::snprintf(conf_name, sizeof conf_name, "%s/conf.%04d", P.config_path, config);
  std::vector<double> conf((size_t)std::max(ntodo, 1) * V3 * 72);
  if (ntodo > 0) {
    int prec = 64;
    st = laph_lime_read_gauge_any(conf_name, LT, L, t0, t0 + ntodo - 1, conf.data(), &prec);
    if (st != LAPH_OK) return die(st, "read gauge");
    if (prec == 32) std::printf("Reading single-precision ILDG data, widened to double\n");
  }
  // timeslices of this process still to solve (all of them without --resume)
  std::vector<int> todo;
  for (int ts = 0; ts < ntodo; ++ts) {
    if (resume && outputs_complete(P.result_path, config, t0 + ts, dim, nev)) {
      std::printf("{\"t\": %d, \"skipped\": \"outputs complete\"}\n", t0 + ts);
      continue;
    }
    todo.push_back(ts);
  }
  const double p1 = P.smear == LAPH_SMEAR_HYP ? P.alpha_1 : (P.smear == LAPH_SMEAR_STOUT ? P.rho : P.alpha);
  const double p2 = P.smear == LAPH_SMEAR_HYP ? P.alpha_2 : 0.0;
  std::vector<double> evals(nev), phases(nev), evec((size_t)dim * nev * 2), vfix((size_t)dim * nev * 2);
  if (phase_reset) std::printf("Resetting old phases is overridden by fix_phase, as in the reference\n");

  if (P.solver == 1) {  // ---- plain: the reference's loop body with the GPU MatShell
    laph_params lp{L, P.LAM_L, P.LAM_C, P.DEG, device};
    laph_ctx* ctx = nullptr;
    st = laph_ctx_create(&ctx, &lp);
    if (st != LAPH_OK) return die(st, "context");
    for (int ts : todo) {
      PetscLogDouble v1, v2;
      PetscTime(&v1);
      st = laph_set_links(ctx, conf.data() + (size_t)ts * V3 * 72, LAPH_LAYOUT_CONF);
      if (st == LAPH_OK) st = laph_smear(ctx, P.smear, p1, p2, P.iter, 1);
      if (st != LAPH_OK) return die(st, "links");
      laph_shell shell{ctx, P.DEG};
      Mat A;
      EPS eps;
      Vec xr, xi;
      PetscErrorCode ierr = MatCreateShell(PETSC_COMM_SELF, PETSC_DECIDE, PETSC_DECIDE, dim, dim, &shell, &A);
      ierr |= MatShellSetOperation(A, MATOP_MULT, (void (*)(void))MatMult_Laplacian2D_GPU);
      ierr |= MatShellSetOperation(A, MATOP_MULT_TRANSPOSE, (void (*)(void))MatMult_Laplacian2D_GPU);
      ierr |= MatShellSetOperation(A, MATOP_GET_DIAGONAL, (void (*)(void))MatGetDiagonal_Laplacian2D_GPU);
      ierr |= MatSetOption(A, MAT_HERMITIAN, PETSC_TRUE);
      ierr |= MatCreateVecs(A, nullptr, &xr);
      ierr |= MatCreateVecs(A, nullptr, &xi);
      ierr |= EPSCreate(PETSC_COMM_SELF, &eps);
      ierr |= EPSSetOperators(eps, A, nullptr);
      ierr |= EPSSetProblemType(eps, EPS_HEP);
      ierr |= EPSSetDimensions(eps, nev, PETSC_DECIDE, PETSC_DECIDE);
      ierr |= EPSSetWhichEigenpairs(eps, EPS_LARGEST_MAGNITUDE);
      ierr |= EPSSetTolerances(eps, P.tol > 0 ? P.tol : 1e-8, PETSC_DEFAULT);
      ierr |= EPSSetFromOptions(eps);
      ierr |= EPSSolve(eps);
      if (ierr) return die(LAPH_EINVAL, "EPS");
      PetscInt nconv;
      EPSGetConverged(eps, &nconv);
      std::vector<double> theta(nev);
      for (PetscInt i = 0; i < nev; ++i) {
        PetscScalar eigr, eigi;
        EPSGetEigenpair(eps, i, &eigr, &eigi, xr, xi);
        PetscScalar* p;
        VecGetArray(xr, &p);
        std::memcpy(evec.data() + (size_t)i * dim * 2, p, sizeof(double) * 2 * dim);
        VecRestoreArray(xr, &p);
        theta[i] = PetscRealPart(eigr);
      }
      laph_fix_phase_host(dim, nev, evec.data(), vfix.data(), phases.data());
      st = laph_write_eigsys_bin(P.result_path, "eigenvectors", config, t0 + ts, dim, nev, vfix.data());
      if (st != LAPH_OK) return die(st, "write eigenvectors");
      laph_recover_spectrum(nev, theta.data(), P.DEG, P.LAM_L, P.LAM_C, evals.data());
      laph_write_eigenvalues_bin(P.result_path, "eigenvalues", config, t0 + ts, nev, evals.data());
      laph_write_eigenvalues_bin(P.result_path, "phases", config, t0 + ts, nev, phases.data());
      PetscTime(&v2);
      std::printf("{\"t\": %d, \"solver\": \"plain\", \"nconv\": %d, \"seconds\": %.4f, \"trace_vdv\": %.12f, "
                  "\"eval0\": %.12f}\n",
                  t0 + ts, nconv, v2 - v1, trace_vdv(dim, nev, vfix.data()), evals[0]);
      EPSDestroy(&eps);
      MatDestroy(&A);
      VecDestroy(&xr);
      VecDestroy(&xi);
    }
    laph_ctx_destroy(ctx);
    return 0;
  }

  // ---- block: every timeslice of this process in one batched solve
  const int nsolve = (int)todo.size();
  if (nsolve == 0) return 0;
  std::vector<laph_problem> probs(nsolve, laph_problem{L, nev});
  laph_solve_opts o;
  laph_solve_opts_default(&o);
  o.smear_kind = P.smear;
  o.smear_p1 = p1;
  o.smear_p2 = p2;
  o.smear_iters = P.iter;
  o.smear_compat = 1;
  o.guard = P.guard;
  o.tol = P.tol > 0 ? P.tol : 1e-9;
  o.window = P.window;
  o.block = P.block;
  o.deg = P.filter_deg > 0 ? P.filter_deg : default_filter_deg(L, o.deg);
  std::vector<float> model;
  if (o.window == LAPH_WINDOW_MLP && !load_window_model(argv[0], &model)) {
    std::fprintf(stderr, "laph_ev_ts: window = mlp but data/window_mlp.bin is missing or invalid\n");
    return 1;
  }
  if (P.autotune > 0) {
    // deg / block / guard from timed solves of the first timeslices, cached beside the results
    const int ns = std::min(nsolve, P.autotune);
    std::vector<const double*> sample(ns);
    for (int i = 0; i < ns; ++i) sample[i] = conf.data() + (size_t)todo[i] * V3 * 72;
    const std::string cache = std::string(P.result_path) + "/laph_autotune.txt";
    laph_tune_result tr;
    st = laph_solver_autotune(probs.data(), nsolve, sample.data(), LAPH_LAYOUT_CONF, ns, &o,
                              model.empty() ? nullptr : model.data(), (int)model.size(), device, cache.c_str(), &tr);
    if (st != LAPH_OK) return die(st, "autotune");
    std::printf("{\"autotune\": {\"deg\": %d, \"block\": %d, \"guard\": %d, \"ms_per_timeslice\": %.3f, "
                "\"trials\": %d, \"from_cache\": %d}}\n",
                tr.deg, tr.block, tr.guard, tr.ms_per_problem, tr.trials, tr.from_cache);
  }
  // waves of as many timeslices as one solver fits in the device's free memory
  // (all of them at 32^3 x 64; about 20 at a time at 48^3 x 96, nev 220)
  int wave = nsolve;
  st = laph_solver_max_batch(probs.data(), nsolve, &o, device, 0.85, &wave);
  if (st != LAPH_OK) return die(st, "device memory");
  if (wave < nsolve)
    std::printf("{\"waves\": %d, \"timeslices_per_wave\": %d}\n", (nsolve + wave - 1) / wave, wave);
  laph_solver* s = nullptr;
  int s_np = 0;
  std::vector<laph_result> res(wave);
  for (int w0 = 0; w0 < nsolve; w0 += wave) {
    const int wn = std::min(wave, nsolve - w0);
    if (wn != s_np) {  // one solver for every full wave, a smaller one for the last
      laph_solver_destroy(s);
      s = nullptr;
      st = laph_solver_create(&s, probs.data() + w0, wn, &o, device);
      if (st != LAPH_OK) return die(st, "solver");
      s_np = wn;
      if (o.window == LAPH_WINDOW_MLP) {
        st = laph_solver_set_window_model(s, model.data(), (int)model.size());
        if (st != LAPH_OK) return die(st, "window model");
      }
    }
    for (int i = 0; i < wn; ++i) {
      st = laph_solver_set_links(s, i, conf.data() + (size_t)todo[w0 + i] * V3 * 72, LAPH_LAYOUT_CONF, 0);
      if (st != LAPH_OK) return die(st, "links");
    }
    st = laph_solver_run(s, res.data());
    if (st != LAPH_OK && st != LAPH_ENOTCONV) return die(st, "solve");
    double ms[4];
    laph_solver_timings(s, ms);
    for (int i = 0; i < wn; ++i) {
      const int ts = todo[w0 + i];
      st = laph_solver_get(s, i, evals.data(), vfix.data(), phases.data(), 0);
      if (st != LAPH_OK) return die(st, "fetch");
      st = laph_write_eigsys_bin(P.result_path, "eigenvectors", config, t0 + ts, dim, nev, vfix.data());
      if (st != LAPH_OK) return die(st, "write eigenvectors");
      laph_write_eigenvalues_bin(P.result_path, "eigenvalues", config, t0 + ts, nev, evals.data());
      laph_write_eigenvalues_bin(P.result_path, "phases", config, t0 + ts, nev, phases.data());
      std::printf("{\"t\": %d, \"solver\": \"block\", \"status\": %d, \"iters\": %d, \"max_resid\": %.3e, "
                  "\"trace_vdv\": %.12f, \"eval0\": %.12f, \"batch_ms\": %.2f}\n",
                  t0 + ts, res[i].status, res[i].iters, res[i].max_resid, res[i].trace_vdv, evals[0], ms[3]);
    }
  }
  laph_solver_destroy(s);
  return 0;
}
