"""The identities the block solver is built on, checked in FP64 numpy on small
random Hermitian operators (no device, no kernels):

1. the correction form of the filter: T_m(B) V = V T_m(Theta_B) + E_m with
   E_0 = 0, E_1 = S / 2, E_{n+1} = 2 B E_n - E_{n-1} + T_n(Theta_B) S and
   S = 2 (B V - V Theta_B), so only E (of the size of the residual) needs the
   low-precision stencil;
2. the Rayleigh-Ritz of the active block against frozen (locked) Ritz
   vectors V_l with A V_l = V_l Theta_l: with G_la = V_l^H W_a and
   H_la = V_l^H A W_a, the projected W'_a = (1 - V_l V_l^H) W_a has
   G' = G_aa - G_la^H G_la and
   H' = H_aa - G_la^H H_la - H_la^H G_la + G_la^H Theta_l G_la,
   and the rotation [-G_la C ; C] of [V_l | W_a] equals W'_a C;
3. the scaled coefficients of both recurrences as the filter kernel applies
   them (Y_j = a_j B X_j + z_j Z_j + g_j S_j per column, FINAL adding
   t_m V_j, with the tables of the solver's coefficient kernel): the
   correction form gives T_m(B) V / nu_m, a direct pass (S = V) gives
   T_{m-1}(B) V / nu_{m-1}, column by column."""
import numpy as np


def _herm(n, rng):
    M = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    return 0.5 * (M + M.conj().T)


def _cheb_diag(theta, m):
    """T_0..T_m of a vector of Ritz values."""
    t = [np.ones_like(theta), theta.copy()]
    for _ in range(m - 1):
        t.append(2 * theta * t[-1] - t[-2])
    return t


def test_filter_correction_form():
    rng = np.random.default_rng(0)
    n, k, m = 60, 8, 12
    B = _herm(n, rng)
    B /= np.abs(np.linalg.eigvalsh(B)).max()  # spectrum in [-1, 1]
    V, _ = np.linalg.qr(rng.normal(size=(n, k)) + 1j * rng.normal(size=(n, k)))
    th = np.real(np.einsum("ij,ij->j", V.conj(), B @ V))  # Ritz values of B on V (any diagonal Theta works)
    S = 2 * (B @ V - V * th[None, :])
    T = _cheb_diag(th, m)
    E_prev, E = np.zeros_like(V), 0.5 * S
    for nn in range(1, m):
        E_prev, E = E, 2 * B @ E - E_prev + T[nn][None, :] * S
    # the direct three-term recurrence of T_m(B) V
    Y_prev, Y = V, B @ V
    for _ in range(m - 1):
        Y_prev, Y = Y, 2 * B @ Y - Y_prev
    W = V * T[m][None, :] + E
    assert np.abs(W - Y).max() <= 1e-12 * np.abs(Y).max()
    # E is of the size of S: with S = 0 (exact eigenvectors) the correction vanishes
    w, X = np.linalg.eigh(B)
    Vx = X[:, :k]
    Sx = 2 * (B @ Vx - Vx * w[None, :k])
    assert np.abs(Sx).max() < 1e-12


def test_frozen_tile_projection_formulas():
    rng = np.random.default_rng(1)
    n, nl, na = 80, 8, 12
    A = _herm(n, rng)
    w, X = np.linalg.eigh(A)
    Vl, thl = X[:, :nl], w[:nl]                        # locked, converged Ritz pairs
    Wa = rng.normal(size=(n, na)) + 1j * rng.normal(size=(n, na))  # the active filtered block
    Gaa, Haa = Wa.conj().T @ Wa, Wa.conj().T @ A @ Wa
    Gla, Hla = Vl.conj().T @ Wa, Vl.conj().T @ A @ Wa
    Gp = Gaa - Gla.conj().T @ Gla
    Hp = Haa - Gla.conj().T @ Hla - Hla.conj().T @ Gla + Gla.conj().T @ (thl[:, None] * Gla)
    Wp = Wa - Vl @ Gla
    assert np.abs(Gp - Wp.conj().T @ Wp).max() < 1e-10
    assert np.abs(Hp - Wp.conj().T @ A @ Wp).max() < 1e-9
    # Rayleigh-Ritz on the projected pencil (H', G'), then the rotation over the whole block
    Lc = np.linalg.cholesky(Gp)
    Mi = np.linalg.inv(Lc).conj().T                    # G' = L L^H, M = L^-H
    th, Q = np.linalg.eigh(Mi.conj().T @ Hp @ Mi)
    C = Mi @ Q
    Vnew = np.hstack([Vl, Wa]) @ np.vstack([-Gla @ C, C])
    assert np.abs(Vnew - Wp @ C).max() < 1e-10
    assert np.abs(Vnew.conj().T @ Vnew - np.eye(na)).max() < 1e-10      # orthonormal
    assert np.abs(Vl.conj().T @ Vnew).max() < 1e-10                     # orthogonal to the frozen vectors
    assert np.abs(Vnew.conj().T @ A @ Vnew - np.diag(th)).max() < 1e-9  # Ritz pairs of A on the active space


def _coef_tables(tb, m, direct):
    """(a, z, g) for steps n = 1..m-1 and the final V coefficient, per column, as the solver's coefficient kernel
    writes them (nu_n = max(1, |T_n(tb)|))."""
    tn = _cheb_diag(tb, m)
    nu = [np.maximum(1.0, np.abs(t)) for t in tn]
    steps = []
    for n in range(1, m):
        if direct:
            a = 1.0 / nu[1] if n == 1 else 2.0 * nu[n - 1] / nu[n]
            z = -nu[n - 2] / nu[n] if n >= 3 else np.zeros_like(tb)
            g = -1.0 / nu[2] if n == 2 else np.zeros_like(tb)
        elif n == 1:
            a, z, g = 1.0 / nu[2], np.zeros_like(tb), tn[1] / nu[2]
        elif n == 2:
            a, z, g = 2.0 * nu[2] / nu[3], np.zeros_like(tb), (tn[2] - 0.5) / nu[3]
        else:
            a, z, g = 2.0 * nu[n] / nu[n + 1], -nu[n - 1] / nu[n + 1], tn[n] / nu[n + 1]
        steps.append((a * np.ones_like(tb), z * np.ones_like(tb), g * np.ones_like(tb)))
    tfin = np.zeros_like(tb) if direct else tn[m] / nu[m]
    return steps, tfin, nu


def _run_filter(B, V, S, steps, tfin):
    """The kernel's step sequence: step 1 reads X = S, step 2 X = Y_1, later X = Y_{n-1} and Z = Y_{n-2}."""
    ys = []
    for n, (a, z, g) in enumerate(steps, start=1):
        X = S if n == 1 else ys[-1]
        Y = a[None, :] * (B @ X) + g[None, :] * S
        if n >= 3:
            Y = Y + z[None, :] * ys[-2]
        ys.append(Y)
    return tfin[None, :] * V + ys[-1]


def test_filter_coefficient_tables_both_forms():
    rng = np.random.default_rng(2)
    n, k, m = 60, 6, 14
    B = _herm(n, rng)
    B /= np.abs(np.linalg.eigvalsh(B)).max()
    V, _ = np.linalg.qr(rng.normal(size=(n, k)) + 1j * rng.normal(size=(n, k)))
    th = np.real(np.einsum("ij,ij->j", V.conj(), B @ V))
    tb = th * 1.3  # mapped Ritz values partly outside [-1, 1], where the scaling matters

    def cheb_apply(deg):
        Y_prev, Y = V, B @ V
        for _ in range(deg - 1):
            Y_prev, Y = Y, 2 * B @ Y - Y_prev
        return Y

    # correction form, Theta_B = diag(tb): W = T_m(B) V / nu_m
    S = 2 * (B @ V - V * tb[None, :])
    steps, tfin, nu = _coef_tables(tb, m, direct=False)
    W = _run_filter(B, V, S, steps, tfin)
    ref = cheb_apply(m) / nu[m][None, :]
    assert np.abs(W - ref).max() <= 1e-11 * np.abs(ref).max()
    # direct pass, S = V: W = T_{m-1}(B) V / nu_{m-1}
    steps, tfin, nu = _coef_tables(tb, m, direct=True)
    W = _run_filter(B, V, V, steps, tfin)
    ref = cheb_apply(m - 1) / nu[m - 1][None, :]
    assert np.abs(W - ref).max() <= 1e-11 * np.abs(ref).max()
