/*
 * laph_matshell.h -- the GPU replacement for the reference's MatShell
 * callbacks (include/shell_matop.h:25-26 of LapH_EigSys).  Written to the
 * real PETSc signatures, so it builds against real PETSc/SLEPc or against
 * petsc_shim.h.  The shell context is a laph_shell (instead of the
 * reference's &V3 plus process-wide singletons): the device-resident
 * timeslice (laph_ctx) and DEG.
 */
#ifndef LAPH_MATSHELL_H_
#define LAPH_MATSHELL_H_
#include "laph_gpu.h"
#ifdef LAPH_USE_REAL_PETSC
#include <slepceps.h>
#else
#include "petsc_shim.h"
#endif

struct laph_shell {
  laph_ctx* ctx; /* links + LAM_L, LAM_C on the device */
  int deg;       /* DEG */
};

/* MatMult_Laplacian2D (modules/shell_matop.cpp:226-244): y = T_DEG(B) x on the
 * GPU, x and y the PETSc Vec host arrays.  As tv_iter, DEG <= 1 leaves y
 * unwritten (shell_matop.cpp:153-167). */
extern "C" PetscErrorCode MatMult_Laplacian2D_GPU(Mat A, Vec x, Vec y);
/* MatGetDiagonal_Laplacian2D (shell_matop.cpp:248-255): -6 everywhere. */
extern "C" PetscErrorCode MatGetDiagonal_Laplacian2D_GPU(Mat A, Vec diag);

#endif
