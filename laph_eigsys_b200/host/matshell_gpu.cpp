// matshell_gpu.cpp -- MatShell callbacks with the product on the GPU: the
// drop-in for MatMult_Laplacian2D / MatGetDiagonal_Laplacian2D
// (modules/shell_matop.cpp:226-255).
#include "../../include/laph_matshell.h"

#include <cstdio>

extern "C" PetscErrorCode MatMult_Laplacian2D_GPU(Mat A, Vec x, Vec y) {
  void* ctx = nullptr;
  const PetscScalar* px;
  PetscScalar* py;
  PetscErrorCode ierr;
  PetscFunctionBeginUser;
  ierr = MatShellGetContext(A, &ctx);
  CHKERRQ(ierr);
  const laph_shell* sh = static_cast<const laph_shell*>(ctx);
  ierr = VecGetArrayRead(x, &px);
  CHKERRQ(ierr);
  ierr = VecGetArray(y, &py);
  CHKERRQ(ierr);
  if (sh->deg >= 2) {  // tv_iter leaves y unwritten for DEG <= 1
    const int st = laph_matmult(sh->ctx, reinterpret_cast<const double*>(px), reinterpret_cast<double*>(py), sh->deg, 0);
    if (st != LAPH_OK) {
      std::fprintf(stderr, "MatMult_Laplacian2D_GPU: %s\n", laph_last_error());
      return st;
    }
  }
  ierr = VecRestoreArrayRead(x, &px);
  CHKERRQ(ierr);
  ierr = VecRestoreArray(y, &py);
  CHKERRQ(ierr);
  PetscFunctionReturn(0);
}

extern "C" PetscErrorCode MatGetDiagonal_Laplacian2D_GPU(Mat A, Vec diag) {
  PetscErrorCode ierr;
  (void)A;
  PetscFunctionBeginUser;
  ierr = VecSet(diag, -6.0);
  CHKERRQ(ierr);
  PetscFunctionReturn(0);
}
