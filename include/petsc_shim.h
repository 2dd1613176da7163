/*
 * petsc_shim.h -- the subset of the PETSc / SLEPc C API that LapH_EigSys's
 * ev_ts uses around its MatShell (src/ev_ts.cpp:128-335), implemented on top
 * of liblaph_gpu.so so that the reference's timeslice loop builds and runs
 * without PETSc/SLEPc.  Where real PETSc/SLEPc are installed, build against
 * them instead: the GPU MatShell callback (laph_matshell.h) is written to
 * the real signatures and drops in unchanged.
 *
 * Semantics kept from PETSc/SLEPc: a MatShell stores a user context and
 * operation callbacks; MatMult calls the MATOP_MULT callback; Vec arrays are
 * contiguous PetscScalar; EPSSolve runs Krylov-Schur (HEP, largest
 * magnitude) with SLEPc's defaults (ncv = max(2 nev, nev + 15), tol 1e-8,
 * max_it = max(100, 2 n / ncv)); EPSSetFromOptions reads -eps_tol,
 * -eps_max_it, -eps_ncv from the PETSC_OPTIONS environment variable, which is
 * how the reference's EPS is tuned (its argv goes to Boost, not PETSc).
 */
#ifndef LAPH_PETSC_SHIM_H_
#define LAPH_PETSC_SHIM_H_
#include <complex>

extern "C" {

typedef int PetscErrorCode;
typedef int PetscInt;
typedef int PetscMPIInt;
typedef double PetscReal;
typedef std::complex<double> PetscScalar;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;
typedef int MPI_Comm;
typedef double PetscLogDouble;
#define PETSC_COMM_SELF 0
#define PETSC_COMM_WORLD 0
#define PETSC_DECIDE (-1)
#define PETSC_DEFAULT (-2)

typedef struct _p_Mat* Mat;
typedef struct _p_Vec* Vec;
typedef struct _p_EPS* EPS;
typedef const char* EPSType;
typedef enum { MATOP_MULT = 0, MATOP_MULT_TRANSPOSE = 1, MATOP_GET_DIAGONAL = 2 } MatOperation;
typedef enum { MAT_HERMITIAN = 0, MAT_SYMMETRIC = 1 } MatOption;
typedef enum { EPS_HEP = 1 } EPSProblemType;
typedef enum { EPS_LARGEST_MAGNITUDE = 1 } EPSWhich;
typedef enum { EPS_CONVERGED_TOL = 1, EPS_DIVERGED_ITS = -1 } EPSConvergedReason;

PetscErrorCode MatCreateShell(MPI_Comm comm, PetscInt m, PetscInt n, PetscInt M, PetscInt N, void* ctx, Mat* A);
PetscErrorCode MatShellSetOperation(Mat A, MatOperation op, void (*f)(void));
PetscErrorCode MatShellGetContext(Mat A, void* ctx); /* ctx: address of a void* */
PetscErrorCode MatSetFromOptions(Mat A);
PetscErrorCode MatSetOption(Mat A, MatOption op, PetscBool flg);
PetscErrorCode MatSetUp(Mat A);
PetscErrorCode MatCreateVecs(Mat A, Vec* right, Vec* left);
PetscErrorCode MatGetSize(Mat A, PetscInt* M, PetscInt* N);
PetscErrorCode MatMult(Mat A, Vec x, Vec y);
PetscErrorCode MatGetDiagonal(Mat A, Vec d);
PetscErrorCode MatDestroy(Mat* A);

PetscErrorCode VecCreateSeq(MPI_Comm comm, PetscInt n, Vec* v);
PetscErrorCode VecGetSize(Vec v, PetscInt* n);
PetscErrorCode VecGetArray(Vec v, PetscScalar** a);
PetscErrorCode VecRestoreArray(Vec v, PetscScalar** a);
PetscErrorCode VecGetArrayRead(Vec v, const PetscScalar** a);
PetscErrorCode VecRestoreArrayRead(Vec v, const PetscScalar** a);
PetscErrorCode VecSet(Vec v, PetscScalar a);
PetscErrorCode VecDestroy(Vec* v);

PetscErrorCode EPSCreate(MPI_Comm comm, EPS* eps);
PetscErrorCode EPSSetOperators(EPS eps, Mat A, Mat B);
PetscErrorCode EPSSetProblemType(EPS eps, EPSProblemType type);
PetscErrorCode EPSSetDimensions(EPS eps, PetscInt nev, PetscInt ncv, PetscInt mpd);
PetscErrorCode EPSSetWhichEigenpairs(EPS eps, EPSWhich which);
PetscErrorCode EPSSetTolerances(EPS eps, PetscReal tol, PetscInt maxits);
PetscErrorCode EPSSetFromOptions(EPS eps);
PetscErrorCode EPSSolve(EPS eps);
PetscErrorCode EPSGetConverged(EPS eps, PetscInt* nconv);
PetscErrorCode EPSGetConvergedReason(EPS eps, EPSConvergedReason* reason);
PetscErrorCode EPSGetIterationNumber(EPS eps, PetscInt* its);
PetscErrorCode EPSGetType(EPS eps, EPSType* type);
PetscErrorCode EPSGetEigenpair(EPS eps, PetscInt i, PetscScalar* eigr, PetscScalar* eigi, Vec xr, Vec xi);
PetscErrorCode EPSDestroy(EPS* eps);

PetscErrorCode PetscTime(PetscLogDouble* t);
PetscErrorCode SlepcInitialize(int* argc, char*** argv, const char* file, const char* help);
PetscErrorCode SlepcFinalize(void);

}  // extern "C"

#define CHKERRQ(e)          \
  do {                      \
    if (e) return (e);      \
  } while (0)
#define PetscFunctionBeginUser
#define PetscFunctionReturn(x) return (x)
#define PetscRealPart(z) ((z).real())

#endif
