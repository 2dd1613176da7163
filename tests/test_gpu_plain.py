"""Plain form: SLEPc-style Krylov-Schur (laph_eps_solve) driving the GPU
MatShell product, host and device Krylov bases, against a dense FP64
eigendecomposition and the oracle's Krylov-Schur; recover_spectrum and
fix_phase applied as in src/ev_ts.cpp:304-319."""
import numpy as np
import pytest

from conftest import random_links

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("device_basis", [False, True])
@pytest.mark.parametrize("L,nev,deg", [(6, 20, 8), (8, 40, 12)])
def test_plain_krylov_schur_matches_dense(gpu, orc, L, nev, deg, device_basis):
    U = orc.smear_hyp(random_links(L, 0.4, 700 + L), L, 0.62, 0.52, 1)
    A = orc.neglap_dense(U, L)
    w = np.linalg.eigvalsh(A)
    lam_l, lam_c = 12.0, 0.5 * (w[nev + 3] + w[nev + 4])
    ctx = gpu.Context(L, lam_l, lam_c, deg)
    ctx.set_links(U)
    st, theta, V, nconv, its, nmv = ctx.eps_solve(nev, tol=1e-12, max_it=200, device_basis=device_basis)
    assert st == 0 and nconv >= nev
    assert np.all(np.diff(np.abs(theta)) <= 1e-9 * np.abs(theta[0]))  # largest magnitude first
    lam = -gpu.recover_spectrum(theta, deg, lam_l, lam_c)  # recover_spectrum stores -lambda
    assert np.abs(np.sort(lam) - w[:nev]).max() < 1e-7
    rq = np.array([np.vdot(V[:, i], A @ V[:, i]).real for i in range(nev)])
    assert np.abs(np.sort(rq) - w[:nev]).max() / w[-1] < 1e-11
    res = np.linalg.norm(A @ V - V * rq[None, :], axis=0) / 12.0
    assert res.max() < 1e-9
    Vf, ph = gpu.fix_phase(V)
    ok, tr, sm = gpu.check_trace(Vf)
    assert ok and abs(tr - nev) < 1e-9
    # same spectrum as the oracle's Krylov-Schur on the same operator
    st2, th2, V2, nc2, its2, nmv2 = orc.eps_solve(U, L, lam_l, lam_c, deg, nev, tol=1e-12)
    assert np.abs(np.sort(theta) - np.sort(th2)).max() / np.abs(th2).max() < 1e-10
    ctx.close()
