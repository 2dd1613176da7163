// petsc_shim.cpp -- the PETSc/SLEPc subset of petsc_shim.h.  Mat is a shell
// (context + operation table), Vec a contiguous PetscScalar array, and
// EPSSolve runs the library's Krylov-Schur (laph_eps_solve_cb) with the
// MatShell's MATOP_MULT as the operator, as SLEPc's EPSSolve does.
#include "../../include/petsc_shim.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/laph_gpu.h"

struct _p_Vec {
  std::vector<PetscScalar> a;
  PetscScalar* view = nullptr;  // non-owning storage when set
  PetscInt n = 0;
  PetscScalar* data() { return view ? view : a.data(); }
};

struct _p_Mat {
  PetscInt M = 0, N = 0;
  void* ctx = nullptr;
  PetscErrorCode (*mult)(Mat, Vec, Vec) = nullptr;
  PetscErrorCode (*mult_t)(Mat, Vec, Vec) = nullptr;
  PetscErrorCode (*diag)(Mat, Vec) = nullptr;
  bool hermitian = false;
};

struct _p_EPS {
  Mat A = nullptr;
  PetscInt nev = 1, ncv = PETSC_DECIDE, max_it = PETSC_DEFAULT;
  PetscReal tol = 1e-8;
  std::vector<double> theta;
  std::vector<PetscScalar> V;
  PetscInt nconv = 0, its = 0;
  int status = 0;
};

extern "C" {

PetscErrorCode MatCreateShell(MPI_Comm, PetscInt, PetscInt, PetscInt M, PetscInt N, void* ctx, Mat* A) {
  if (!A || M <= 0 || N <= 0) return 1;
  *A = new _p_Mat();
  (*A)->M = M;
  (*A)->N = N;
  (*A)->ctx = ctx;
  return 0;
}

PetscErrorCode MatShellSetOperation(Mat A, MatOperation op, void (*f)(void)) {
  if (!A) return 1;
  if (op == MATOP_MULT) A->mult = reinterpret_cast<PetscErrorCode (*)(Mat, Vec, Vec)>(f);
  else if (op == MATOP_MULT_TRANSPOSE) A->mult_t = reinterpret_cast<PetscErrorCode (*)(Mat, Vec, Vec)>(f);
  else if (op == MATOP_GET_DIAGONAL) A->diag = reinterpret_cast<PetscErrorCode (*)(Mat, Vec)>(f);
  else return 1;
  return 0;
}

PetscErrorCode MatShellGetContext(Mat A, void* ctx) {
  if (!A || !ctx) return 1;
  *static_cast<void**>(ctx) = A->ctx;
  return 0;
}

PetscErrorCode MatSetFromOptions(Mat A) { return A ? 0 : 1; }
PetscErrorCode MatSetOption(Mat A, MatOption op, PetscBool flg) {
  if (!A) return 1;
  if (op == MAT_HERMITIAN) A->hermitian = flg == PETSC_TRUE;
  return 0;
}
PetscErrorCode MatSetUp(Mat A) { return A ? 0 : 1; }

PetscErrorCode VecCreateSeq(MPI_Comm, PetscInt n, Vec* v) {
  if (!v || n < 0) return 1;
  *v = new _p_Vec();
  (*v)->a.assign(n, PetscScalar(0.0));
  (*v)->n = n;
  return 0;
}

PetscErrorCode MatCreateVecs(Mat A, Vec* right, Vec* left) {
  if (!A) return 1;
  if (right && VecCreateSeq(0, A->N, right)) return 1;
  if (left && VecCreateSeq(0, A->M, left)) return 1;
  return 0;
}

PetscErrorCode MatGetSize(Mat A, PetscInt* M, PetscInt* N) {
  if (!A) return 1;
  if (M) *M = A->M;
  if (N) *N = A->N;
  return 0;
}

PetscErrorCode MatMult(Mat A, Vec x, Vec y) {
  if (!A || !A->mult || !x || !y) return 1;
  return A->mult(A, x, y);
}

PetscErrorCode MatGetDiagonal(Mat A, Vec d) {
  if (!A || !A->diag || !d) return 1;
  return A->diag(A, d);
}

PetscErrorCode MatDestroy(Mat* A) {
  if (A && *A) {
    delete *A;
    *A = nullptr;
  }
  return 0;
}

PetscErrorCode VecGetSize(Vec v, PetscInt* n) {
  if (!v || !n) return 1;
  *n = v->n;
  return 0;
}
PetscErrorCode VecGetArray(Vec v, PetscScalar** a) {
  if (!v || !a) return 1;
  *a = v->data();
  return 0;
}
PetscErrorCode VecRestoreArray(Vec v, PetscScalar** a) { return v && a ? 0 : 1; }
PetscErrorCode VecGetArrayRead(Vec v, const PetscScalar** a) {
  if (!v || !a) return 1;
  *a = v->data();
  return 0;
}
PetscErrorCode VecRestoreArrayRead(Vec v, const PetscScalar** a) { return v && a ? 0 : 1; }
PetscErrorCode VecSet(Vec v, PetscScalar s) {
  if (!v) return 1;
  PetscScalar* p = v->data();
  for (PetscInt i = 0; i < v->n; ++i) p[i] = s;
  return 0;
}
PetscErrorCode VecDestroy(Vec* v) {
  if (v && *v) {
    delete *v;
    *v = nullptr;
  }
  return 0;
}

PetscErrorCode EPSCreate(MPI_Comm, EPS* eps) {
  if (!eps) return 1;
  *eps = new _p_EPS();
  return 0;
}
PetscErrorCode EPSSetOperators(EPS eps, Mat A, Mat B) {
  if (!eps || !A || B) return 1;  // standard problems only
  eps->A = A;
  return 0;
}
PetscErrorCode EPSSetProblemType(EPS eps, EPSProblemType type) { return eps && type == EPS_HEP ? 0 : 1; }
PetscErrorCode EPSSetDimensions(EPS eps, PetscInt nev, PetscInt ncv, PetscInt) {
  if (!eps || nev < 1) return 1;
  eps->nev = nev;
  eps->ncv = ncv;
  return 0;
}
PetscErrorCode EPSSetWhichEigenpairs(EPS eps, EPSWhich which) { return eps && which == EPS_LARGEST_MAGNITUDE ? 0 : 1; }
PetscErrorCode EPSSetTolerances(EPS eps, PetscReal tol, PetscInt maxits) {
  if (!eps) return 1;
  if (tol != PETSC_DEFAULT) eps->tol = tol;
  if (maxits != PETSC_DEFAULT) eps->max_it = maxits;
  return 0;
}

// -eps_tol / -eps_max_it / -eps_ncv from PETSC_OPTIONS
PetscErrorCode EPSSetFromOptions(EPS eps) {
  if (!eps) return 1;
  const char* env = std::getenv("PETSC_OPTIONS");
  if (!env) return 0;
  std::string s(env);
  auto val = [&](const char* key, std::string* out) {
    const size_t p = s.find(key);
    if (p == std::string::npos) return false;
    size_t q = p + std::strlen(key);
    while (q < s.size() && s[q] == ' ') ++q;
    size_t e = q;
    while (e < s.size() && s[e] != ' ') ++e;
    *out = s.substr(q, e - q);
    return !out->empty();
  };
  std::string v;
  if (val("-eps_tol", &v)) eps->tol = std::atof(v.c_str());
  if (val("-eps_max_it", &v)) eps->max_it = std::atoi(v.c_str());
  if (val("-eps_ncv", &v)) eps->ncv = std::atoi(v.c_str());
  return 0;
}

namespace {
// MATOP_MULT on raw host arrays, through Vec views
int shell_mult(void* user, const double* x, double* y) {
  Mat A = static_cast<Mat>(user);
  _p_Vec vx, vy;
  vx.view = reinterpret_cast<PetscScalar*>(const_cast<double*>(x));
  vx.n = A->N;
  vy.view = reinterpret_cast<PetscScalar*>(y);
  vy.n = A->M;
  return A->mult(A, &vx, &vy);
}
}  // namespace

PetscErrorCode EPSSolve(EPS eps) {
  if (!eps || !eps->A || !eps->A->mult) return 1;
  const long long n = eps->A->N;
  const int ncv = eps->ncv > 0 ? eps->ncv : 0;
  const int m = ncv > 0 ? ncv : std::max(2 * eps->nev, eps->nev + 15);
  const int max_it = eps->max_it > 0 ? eps->max_it : std::max(100, (int)(2 * n / std::max(1, m)));
  eps->theta.assign(eps->nev, 0.0);
  eps->V.assign((size_t)n * eps->nev, PetscScalar(0.0));
  int nconv = 0, its = 0;
  long long nmv = 0;
  eps->status = laph_eps_solve_cb(n, shell_mult, eps->A, eps->nev, ncv, eps->tol, max_it, 0x12345678ULL,
                                  eps->theta.data(), reinterpret_cast<double*>(eps->V.data()), &nconv, &its, &nmv);
  eps->nconv = nconv;
  eps->its = its;
  // SLEPc reports non-convergence through the converged reason, not an error
  return (eps->status == LAPH_OK || eps->status == LAPH_ENOTCONV) ? 0 : eps->status;
}

PetscErrorCode EPSGetConverged(EPS eps, PetscInt* nconv) {
  if (!eps || !nconv) return 1;
  *nconv = eps->nconv;
  return 0;
}
PetscErrorCode EPSGetConvergedReason(EPS eps, EPSConvergedReason* r) {
  if (!eps || !r) return 1;
  *r = eps->status == LAPH_OK ? EPS_CONVERGED_TOL : EPS_DIVERGED_ITS;
  return 0;
}
PetscErrorCode EPSGetIterationNumber(EPS eps, PetscInt* its) {
  if (!eps || !its) return 1;
  *its = eps->its;
  return 0;
}
PetscErrorCode EPSGetType(EPS eps, EPSType* type) {
  if (!eps || !type) return 1;
  *type = "krylovschur";
  return 0;
}
PetscErrorCode EPSGetEigenpair(EPS eps, PetscInt i, PetscScalar* eigr, PetscScalar* eigi, Vec xr, Vec xi) {
  if (!eps || i < 0 || i >= (PetscInt)eps->theta.size()) return 1;
  if (eigr) *eigr = eps->theta[i];
  if (eigi) *eigi = 0.0;
  const size_t n = eps->A->N;
  if (xr) std::memcpy(static_cast<void*>(xr->data()), &eps->V[(size_t)i * n], n * sizeof(PetscScalar));
  if (xi) VecSet(xi, 0.0);
  return 0;
}
PetscErrorCode EPSDestroy(EPS* eps) {
  if (eps && *eps) {
    delete *eps;
    *eps = nullptr;
  }
  return 0;
}

PetscErrorCode PetscTime(PetscLogDouble* t) {
  *t = std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
  return 0;
}
PetscErrorCode SlepcInitialize(int*, char***, const char*, const char*) { return 0; }
PetscErrorCode SlepcFinalize(void) { return 0; }

}  // extern "C"
