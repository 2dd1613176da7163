"""Covariant displacement (right_displacement_one_dir): the device kernel against
the oracle, anti-Hermiticity, gauge covariance, and the solver's in-place path."""
import numpy as np
import pytest

import laph_eigsys_b200 as lb
from conftest import pure_gauge_links, random_links, random_su3_field, unit_links


def test_oracle_displacement_properties(orc):
    L = 4
    U = random_links(L, 0.4, 9)
    rng = np.random.default_rng(2)
    V = rng.normal(size=(3 * L ** 3, 4)) + 1j * rng.normal(size=(3 * L ** 3, 4))
    for d in range(3):
        W = orc.displace(U, L, d, V)
        # D is anti-Hermitian: <a, D b> = -<D a, b>
        assert abs(np.vdot(V[:, 0], W[:, 1]) + np.vdot(W[:, 0], V[:, 1])) < 1e-12
    # unit links: D = (shift_up - shift_down) / 2 annihilates constant fields
    W = orc.displace(unit_links(L), L, 2, np.ones((3 * L ** 3, 1), dtype=np.complex128))
    assert np.abs(W).max() < 1e-15
    # gauge covariance: U -> Omega(x)^dag U Omega(x+mu) (pure gauge), v -> Omega^dag v
    Om = random_su3_field(L, 4)
    Ug = pure_gauge_links(L, Om)
    v = np.ones((L ** 3, 3), dtype=np.complex128)
    vg = np.einsum("sba,sb->sa", Om.conj(), v).reshape(-1, 1)  # Omega(x)^dag v(x)
    Wg = orc.displace(Ug, L, 0, vg).reshape(L ** 3, 3)
    W1 = orc.displace(unit_links(L), L, 0, v.reshape(-1, 1)).reshape(L ** 3, 3)
    assert np.abs(Wg - np.einsum("sba,sb->sa", Om.conj(), W1)).max() < 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("L,nev", [(4, 5), (6, 20), (8, 33)])
def test_displace_kernel_matches_oracle(gpu, orc, L, nev):
    U = random_links(L, 0.4, 40 + L)
    rng = np.random.default_rng(L)
    V = rng.normal(size=(3 * L ** 3, nev)) + 1j * rng.normal(size=(3 * L ** 3, nev))
    ctx = gpu.Context(L)
    ctx.set_links(U)
    for d in range(3):
        W = ctx.displace(V, d)
        R = orc.displace(U, L, d, V)
        assert np.abs(W - R).max() <= 1e-14 * np.abs(R).max()
    ctx.close()


@pytest.mark.gpu
def test_solver_displace_smeared_eigenvectors(gpu, orc):
    """Problem i's phase-fixed eigenvectors displaced with its smeared links, in place on the device."""
    L, nev = 6, 12
    U = random_links(L, 0.4, 51)
    s = gpu.Solver([(L, nev), (4, 6)], tol=1e-10, deg=8, max_it=300, smear_kind=gpu.SMEAR_STOUT, smear_p1=0.1,
                   smear_iters=2, smear_compat=1)
    s.set_links(0, U)
    s.set_links(1, random_links(4, 0.4, 52))
    st, _ = s.run()
    assert st == 0
    _, V, _ = s.get(0)
    Us = orc.smear_stout(U, L, 0.1, 2, 1)
    for d in range(3):
        W = s.displace(0, d)
        R = orc.displace(Us, L, d, V)
        assert np.abs(W - R).max() <= 1e-13 * np.abs(R).max()
    s.close()
