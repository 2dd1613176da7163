"""The PETSc/SLEPc-shaped host layer on CPU: a MatShell whose MATOP_MULT is a
host callback (here the oracle's tv_iter, T_DEG(B) of the reference), driven
by the shim's EPSSolve (the library's Krylov-Schur) exactly as ev_ts drives
SLEPc -- no device needed.  Eigenpairs against a dense eigendecomposition."""
import ctypes
import os

import numpy as np

from conftest import random_links

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "laph_eigsys_b200", "libpetsc_shim.so")

MATOP_MULT, MAT_HERMITIAN, EPS_HEP, EPS_LARGEST_MAGNITUDE, PETSC_DECIDE = 0, 0, 1, 1, -1
c_vp, c_int = ctypes.c_void_p, ctypes.c_int
CB = ctypes.CFUNCTYPE(c_int, c_vp, c_vp, c_vp)


def test_shim_eps_solves_matshell_like_slepc(orc):
    shim = ctypes.CDLL(SHIM)
    L, nev, deg, lam_l = 4, 12, 8, 12.0
    U = orc.smear_hyp(random_links(L, 0.4, 99), L, 0.62, 0.52, 1)
    A = orc.neglap_dense(U, L)
    w = np.linalg.eigvalsh(A)
    lam_c = 0.5 * (w[nev + 2] + w[nev + 3])
    dim = 3 * L ** 3
    calls = [0]

    def mult(Amat, x, y):
        px, py = c_vp(), c_vp()
        shim.VecGetArrayRead(c_vp(x), ctypes.byref(px))
        shim.VecGetArray(c_vp(y), ctypes.byref(py))
        xv = np.ctypeslib.as_array(ctypes.cast(px, ctypes.POINTER(ctypes.c_double)), (2 * dim,)).view(np.complex128)
        yv = np.ctypeslib.as_array(ctypes.cast(py, ctypes.POINTER(ctypes.c_double)), (2 * dim,)).view(np.complex128)
        yv[:] = orc.tv_iter(U, L, lam_l, lam_c, deg, xv.copy())
        calls[0] += 1
        return 0

    cb = CB(mult)
    Am, eps, xr, xi = c_vp(), c_vp(), c_vp(), c_vp()
    assert shim.MatCreateShell(0, PETSC_DECIDE, PETSC_DECIDE, dim, dim, None, ctypes.byref(Am)) == 0
    assert shim.MatShellSetOperation(Am, MATOP_MULT, ctypes.cast(cb, c_vp)) == 0
    assert shim.MatSetOption(Am, MAT_HERMITIAN, 1) == 0
    assert shim.MatCreateVecs(Am, None, ctypes.byref(xr)) == 0
    assert shim.MatCreateVecs(Am, None, ctypes.byref(xi)) == 0
    assert shim.EPSCreate(0, ctypes.byref(eps)) == 0
    assert shim.EPSSetOperators(eps, Am, None) == 0
    assert shim.EPSSetProblemType(eps, EPS_HEP) == 0
    assert shim.EPSSetDimensions(eps, nev, PETSC_DECIDE, PETSC_DECIDE) == 0
    assert shim.EPSSetWhichEigenpairs(eps, EPS_LARGEST_MAGNITUDE) == 0
    shim.EPSSetTolerances.argtypes = [c_vp, ctypes.c_double, c_int]
    assert shim.EPSSetTolerances(eps, 1e-12, -2) == 0
    assert shim.EPSSolve(eps) == 0
    nconv = c_int()
    shim.EPSGetConverged(eps, ctypes.byref(nconv))
    assert nconv.value >= nev and calls[0] > 0
    eig = (ctypes.c_double * 2)()
    rq = []
    for i in range(nev):
        assert shim.EPSGetEigenpair(eps, i, eig, None, xr, xi) == 0
        p = c_vp()
        shim.VecGetArray(xr, ctypes.byref(p))
        v = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_double)), (2 * dim,)).view(np.complex128).copy()
        rq.append(np.vdot(v, A @ v).real)
    assert np.abs(np.sort(rq) - w[:nev]).max() / w[-1] < 1e-11
    shim.EPSDestroy(ctypes.byref(eps))
    shim.MatDestroy(ctypes.byref(Am))
