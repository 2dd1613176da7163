"""Oracle pins: analytic known answers derived from the reference's own checks
(unit gauge field, pure gauge, SU(3), tr(V^dag V) = nev, dense -Delta)."""
import numpy as np
import pytest

from conftest import pure_gauge_links, random_links, random_su3_field, unit_links


def su3_err(U):
    M = U.reshape(-1, 3, 3)
    uu = np.conj(np.transpose(M, (0, 2, 1))) @ M
    return max(np.abs(uu - np.eye(3)).max(), np.abs(np.linalg.det(M) - 1).max())


def test_gauge_random_is_su3():
    U = random_links(4, 0.4, 1227)
    assert su3_err(U) < 1e-13


def test_proj_su3_matches_polar_decomposition(orc):
    rng = np.random.default_rng(5)
    for _ in range(20):
        M = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
        W = orc.proj_su3(M)
        # polar factor via SVD, then det^{-1/3} on the principal branch
        u, s, vh = np.linalg.svd(M)
        P = u @ vh
        d = np.linalg.det(P)
        P = P / d ** (1.0 / 3.0)
        assert np.abs(W - P).max() < 1e-12
        assert su3_err(W) < 1e-13


def test_expiH(orc):
    rng = np.random.default_rng(2)
    A = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
    H = A + A.conj().T
    w, Q = np.linalg.eigh(H)
    ref = Q @ np.diag(np.exp(1j * w)) @ Q.conj().T
    assert np.abs(orc.expiH(H) - ref).max() < 1e-13


@pytest.mark.parametrize("kind", ["stout", "ape", "hyp"])
def test_unit_field_is_fixed_point_of_smearing(orc, kind):
    L = 4
    U = unit_links(L)
    if kind == "stout":
        S = orc.smear_stout(U, L, 0.1, 3)
    elif kind == "ape":
        S = orc.smear_ape(U, L, 0.5, 3)
    else:
        S = orc.smear_hyp(U, L, 0.62, 0.52, 3)
    assert np.abs(S - U).max() < 1e-14


@pytest.mark.parametrize("L", [4, 6])
def test_free_spectrum_from_krylov_schur(orc, L):
    """Unit gauge field: every converged pair lies on the analytic spectrum
    sum_i 4 sin^2(pi n_i/L) (x3 colours), the lowest being the 3 zero modes.
    (A single-vector Krylov method resolves massively degenerate eigenvalues
    only through rounding, as SLEPc's does, so multiplicities are not pinned.)"""
    U = unit_links(L)
    nev = 12
    lam_l, lam_c, deg = 12.5, 3.0, 8
    st, theta, V, nconv, its, nmv = orc.eps_solve(U, L, lam_l, lam_c, deg, nev, tol=1e-13)
    ref = np.unique(np.round(orc.free_spectrum(L), 12))
    ok = theta >= 1.0
    assert ok.sum() >= 3
    lam = -orc.recover_spectrum(theta[ok], deg, lam_l, lam_c)
    assert np.abs(lam[:, None] - ref[None, :]).min(axis=1).max() < 1e-9
    rq = np.array([np.vdot(V[:, i], orc.neglap(U, L, V[:, i])).real for i in np.flatnonzero(ok)])
    assert np.abs(rq[:, None] - ref[None, :]).min(axis=1).max() < 1e-11
    assert np.abs(np.sort(rq)[:3]).max() < 1e-11


def test_dense_spectrum_random_field(orc):
    L = 4
    U = orc.smear_stout(random_links(L, 0.4, 1227), L, 0.1, 3)
    A = orc.neglap_dense(U, L)
    assert np.abs(A - A.conj().T).max() < 1e-14
    w = np.linalg.eigvalsh(A)
    nev = 24
    lam_c = 0.5 * (w[nev + 4] + w[nev + 5])
    lam_l, deg = 12.5, 8
    st, theta, V, nconv, its, nmv = orc.eps_solve(U, L, lam_l, lam_c, deg, nev, tol=1e-13)
    assert st == 0
    rq = np.sort([np.vdot(V[:, i], A @ V[:, i]).real for i in range(nev)])
    assert np.abs(rq - w[:nev]).max() / w[-1] < 1e-11
    lam = np.sort(-orc.recover_spectrum(theta, deg, lam_l, lam_c))
    assert np.abs(lam - w[:nev]).max() < 1e-7  # recover_spectrum loses digits near theta ~ 1
    VdV = V.conj().T @ V
    assert abs(np.trace(VdV).real - nev) < 1e-9


def test_tv_iter_is_chebyshev_polynomial(orc):
    L = 4
    U = random_links(L, 0.4, 1228)
    A = orc.neglap_dense(U, L)
    lam_l, lam_c = 11.8, 0.6
    c = 2.0 / (lam_l - lam_c)
    a = 1 + c * lam_c
    B = a * np.eye(A.shape[0]) - c * A
    rng = np.random.default_rng(0)
    x = rng.normal(size=A.shape[0]) + 1j * rng.normal(size=A.shape[0])
    assert np.abs(orc.tv2(U, L, lam_l, lam_c, x) - B @ x).max() < 1e-12
    Tm, T = x, B @ x
    for n in range(2, 9):
        Tm, T = T, 2 * B @ T - Tm
        y = orc.tv_iter(U, L, lam_l, lam_c, n, x)
        assert np.abs(y - T).max() / np.abs(T).max() < 1e-12
    # deg <= 1 leaves y unwritten (shell_matop.cpp:153-167)
    y0 = np.full_like(x, 7.0)
    assert np.array_equal(orc.tv_iter(U, L, lam_l, lam_c, 1, x, y0), y0)


def test_pure_gauge_covariance(orc):
    """U = Omega^dag(x) Omega(x+mu): -Delta is unitarily equivalent to the free one;
    HYP keeps the field pure gauge, the reference's stout/APE staple quirk does not."""
    L = 4
    Om = random_su3_field(L, 77)
    U = pure_gauge_links(L, Om)
    A = orc.neglap_dense(U, L)
    assert np.abs(np.linalg.eigvalsh(A) - orc.free_spectrum(L)).max() < 1e-12
    H = orc.smear_hyp(U, L, 0.62, 0.52, 2)
    assert np.abs(H - U).max() < 1e-12
    S_ok = orc.smear_stout(U, L, 0.1, 1, compat=0)
    assert np.abs(S_ok - U).max() < 1e-12
    S_q = orc.smear_stout(U, L, 0.1, 1, compat=1)
    assert np.abs(S_q - U).max() > 1e-3


def test_fix_phase(orc):
    rng = np.random.default_rng(3)
    V = rng.normal(size=(48, 5)) + 1j * rng.normal(size=(48, 5))
    Vf, ph = orc.fix_phase(V)
    assert np.abs(Vf[0].imag).max() < 1e-15 and (Vf[0].real >= 0).all()
    assert np.allclose(ph, np.angle(V[0]))
    assert np.allclose(np.abs(Vf), np.abs(V))


def test_plaquette_unit_and_random(orc):
    assert abs(orc.plaquette(unit_links(4), 4) - 1.0) < 1e-15
    U = random_links(4, 0.4, 1227)
    p0 = orc.plaquette(U, 4)
    p1 = orc.plaquette(orc.smear_hyp(U, 4, 0.62, 0.62, 1), 4)
    assert p1 > p0  # smearing raises the plaquette


@pytest.mark.parametrize("cond", [1e2, 1e4, 1e6])
def test_proj_su3_ill_conditioned(orc, cond):
    """The projection's Jacobi route (the one the device kernel shares) on matrices with singular values spread
    over `cond`, and on near-unitary ones (what smearing produces).  The reference's formula M (M^dag M)^{-1/2}
    squares the condition number, so its polar factor is good to ~cond^2 eps (numpy's eigh on the same formula does
    no better), and so is the unitarity of the result; near-unitary inputs come out at rounding level."""
    rng = np.random.default_rng(int(np.log10(cond)))
    for _ in range(20):
        u, _ = np.linalg.qr(rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3)))
        v, _ = np.linalg.qr(rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3)))
        M = u @ np.diag([1.0, cond ** -0.5, 1.0 / cond]) @ v
        W = orc.proj_su3(M)
        P = u @ v
        P = P / np.linalg.det(P) ** (1.0 / 3.0)
        bound = 100 * cond ** 2 * 2.2e-16 + 1e-12
        assert np.abs(W - P).max() < bound and su3_err(W) < bound
        N = P + 1e-3 * (rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3)))  # near-unitary
        u2, s2, vh2 = np.linalg.svd(N)
        Q = u2 @ vh2
        Q = Q / np.linalg.det(Q) ** (1.0 / 3.0)
        assert np.abs(orc.proj_su3(N) - Q).max() < 1e-13


def test_oracle_gauge_generator_matches_the_library(orc):
    """The oracle's restatement of the seeded field generator (used where the library must not be loaded, such as
    the CPU reference arm) gives the library's field to rounding, SU(3) link by link."""
    import laph_eigsys_b200 as lb
    a = orc.gauge_random(5, 3, 0.3, 1229)
    b = lb.gauge_random(5, 3, 0.3, 1229)
    assert np.abs(a - b).max() < 1e-13
    U = a.reshape(-1, 3, 3)
    assert np.abs(U @ np.conj(np.transpose(U, (0, 2, 1))) - np.eye(3)).max() < 1e-13
    assert np.abs(np.linalg.det(U) - 1.0).max() < 1e-13
