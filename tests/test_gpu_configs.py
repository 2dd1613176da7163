"""Parity at the benchmark configurations, against the FP64 oracle,
with every error stated (printed) as well as bounded:

  C1  8^3 x 16, eps 0.4, seed 1227, stout 3 x 0.1 (the reference's backward
      staple), nev 60: all 16 timeslices in one batch against the oracle's
      smearing and a dense eigendecomposition of the assembled -Delta (dim
      1536), and timeslice 0 also against the oracle's Krylov-Schur on
      T_8(B) (the reference's EPSSolve, src/ev_ts.cpp:231-263).
  C2  24^3, eps 0.3, seed 1228, HYP 0.62 / 0.62 x 1, nev 120: timeslices 0
      and 1 against the oracle's smearing + FP64 Krylov-Schur on T_12(B).
  C3  32^3, eps 0.3, seed 1229, stout 5 x 0.1, nev 120, with the BF16 +
      per-site-scale filter links that configuration specifies, C4's 32^3
      lattice (seed 1232, APE 0.5 x 10, nev 180) and C5's 48^3 lattice
      (seed 1233, eps 0.25, stout 6 x 0.1, nev 220, learned window): a
      timeslice each at the configurations' tolerance 1e-9 against the
      oracle's Krylov-Schur.

The block solver's filter runs in FP32 (FP64 Rayleigh-Ritz); its errors are
those of the FP32-filter path against the FP64 oracle.  Eigenvalues are FP64
Rayleigh quotients on -Delta, compared each relative to itself (<= 1e-10) and
relative to lambda_max (<= 1e-10).  At the configurations' tolerance 1e-9 the
eigenvalues and residuals are checked; eigenvectors are determined only to
about residual / gap, so they are compared in a second solve at tolerance
1e-12: phase-fixed vectors of eigenvalues isolated by 0.01 or more, and
subspaces (sin of the largest principal angle) of the clusters closer than
that, both <= 1e-8; tr(V^dag V) = nev to 1e-9."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GAP = 1e-2


def _links(gpu, L, T, eps, seed, ts):
    conf = gpu.gauge_random(L, T, eps, seed)
    return [np.ascontiguousarray(conf[t, :, 1:4]) for t in ts]


def _solve(gpu, L, nev, links, tol, deg, **smear):
    s = gpu.Solver([(L, nev)] * len(links), guard=16, tol=tol, deg=deg, max_it=400, link_prec=gpu.LINKS_FP32,
                   window=gpu.WINDOW_LANCZOS, **smear)
    for i, U in enumerate(links):
        s.set_links(i, U)
    st, res = s.run()
    out = [(s.get(i), s.ritz(i)) for i in range(len(links))]
    s.close()
    assert st == 0, res
    return out


def _check(orc, Us, L, V, Vo, lam_next, tol, vectors, label):
    r = orc.compare_eigensystems(Us, L, V, Vo, gap=GAP, lam_next=lam_next)
    print(label, {k: (f"{v:.2e}" if isinstance(v, float) else v) for k, v in r.items()})
    assert r["max_rel_eig"] <= 1e-10
    assert r["max_eig_over_lam_max"] <= 1e-10
    assert r["max_resid_checked"] <= tol * 1.01
    assert abs(r["trace_vdv_checked"] - r["nev"]) <= 1e-9
    if vectors:
        assert r["max_vec_phase_fixed"] <= 1e-8
        assert r["max_cluster_proj"] <= 1e-8
    return r


def test_c1_all_timeslices_against_dense(gpu, orc):
    L, T, nev = 8, 16, 60
    links = _links(gpu, L, T, 0.4, 1227, range(T))
    smear = dict(smear_kind=gpu.SMEAR_STOUT, smear_p1=0.1, smear_iters=3, smear_compat=1)
    ref = []
    for U in links:
        Us = orc.smear_stout(U, L, 0.1, 3, 1)
        w, X = np.linalg.eigh(orc.neglap_dense(Us, L))
        Xf, _ = orc.fix_phase(X[:, :nev])
        ref.append((Us, w, Xf))
    # the smeared links themselves, through the context (<= 1e-12 per link)
    ctx = gpu.Context(L)
    for U, (Us, _, _) in zip(links, ref):
        ctx.set_links(U)
        ctx.smearing_stout(0.1, 3, 1)
        got = ctx.get_links().reshape(-1, 9)
        err = (np.linalg.norm(got - Us.reshape(-1, 9), axis=1) / np.linalg.norm(Us.reshape(-1, 9), axis=1)).max()
        assert err <= 1e-12
    ctx.close()
    for tol, vectors in ((1e-9, False), (1e-12, True)):
        out = _solve(gpu, L, nev, links, tol, 32, **smear)
        for t, ((ev, V, _), ritz) in enumerate(out):
            Us, w, Xf = ref[t]
            assert np.abs(-ev - w[:nev]).max() <= 1e-10 * 12
            _check(orc, Us, L, V, Xf, w[nev], tol, vectors, f"c1 t={t} tol={tol}")


def test_c1_timeslice0_against_krylov_schur(gpu, orc):
    """The reference's own algorithm on C1's timeslice 0: Krylov-Schur on T_8(B), LAM_L 12, LAM_C above lambda_60
    (2.07), tol 1e-13, its eigenvectors phase-fixed; the block solver at 1e-12 agrees with it as with eigh."""
    L, nev = 8, 60
    U = _links(gpu, L, 16, 0.4, 1227, [0])[0]
    Us = orc.smear_stout(U, L, 0.1, 3, 1)
    st, theta, Vk, nconv, _, _ = orc.eps_solve(Us, L, 12.0, 2.07, 8, nev, tol=1e-13, max_it=400)
    assert st == 0 and nconv >= nev
    Vo, _ = orc.fix_phase(Vk)
    (ev, V, _), ritz = _solve(gpu, L, nev, [U], 1e-12, 32, smear_kind=gpu.SMEAR_STOUT, smear_p1=0.1,
                              smear_iters=3, smear_compat=1)[0]
    _check(orc, Us, L, V, Vo, ritz[nev], 1e-12, True, "c1 t=0 vs Krylov-Schur")


@pytest.mark.parametrize("tol,vectors", [(1e-9, False), (1e-12, True)])
def test_c2_against_krylov_schur(gpu, orc, tol, vectors):
    L, nev = 24, 120
    links = _links(gpu, L, 2, 0.3, 1228, [0, 1])
    out = _solve(gpu, L, nev, links, tol, 60, smear_kind=gpu.SMEAR_HYP, smear_p1=0.62, smear_p2=0.62, smear_iters=1)
    orc.set_threads(os.cpu_count() or 1)
    for t, ((ev, V, _), ritz) in enumerate(out):
        Us = orc.smear_hyp(links[t], L, 0.62, 0.62, 1)
        lam_c = float(1.1 * (-ev)[-1])  # above lambda_120, as a run of the reference would set LAM_C
        st, _, Vk, nconv, _, _ = orc.eps_solve(Us, L, 12.0, lam_c, 12, nev, tol=1e-13, max_it=400)
        assert st == 0 and nconv >= nev
        Vo, _ = orc.fix_phase(Vk)
        _check(orc, Us, L, V, Vo, ritz[nev], tol, vectors, f"c2 t={t} tol={tol}")


@pytest.mark.parametrize("case", ["c3_bf16", "c4_32", "c5_48"])
def test_headline_volume_against_krylov_schur(gpu, orc, case):
    """32^3 and 48^3 timeslices at the configuration tolerance 1e-9, each against the oracle's smearing + FP64
    Krylov-Schur on T_12(B) (tol 1e-10): eigenvalues (FP64 Rayleigh quotients) to 1e-10 relative each and of
    lambda_max, residuals at the tolerance, tr(V^dag V) = nev, and the nev-block subspace to the residual over the
    gap.  C5 (48^3, eps 0.25, stout 6 x 0.1, nev 220) runs with the learned window it specifies."""
    L, eps, window = 32, 0.3, gpu.WINDOW_LANCZOS
    if case == "c3_bf16":
        nev, seed, kind, p1, iters = 120, 1229, gpu.SMEAR_STOUT, 0.1, 5
        prec = gpu.LINKS_BF16
    elif case == "c4_32":
        nev, seed, kind, p1, iters = 180, 1232, gpu.SMEAR_APE, 0.5, 10
        prec = gpu.LINKS_FP32
    else:
        L, eps, window = 48, 0.25, gpu.WINDOW_MLP
        nev, seed, kind, p1, iters = 220, 1233, gpu.SMEAR_STOUT, 0.1, 6
        prec = gpu.LINKS_FP32
    U = _links(gpu, L, 1, eps, seed, [0])[0]
    s = gpu.Solver([(L, nev)], guard=16, tol=1e-9, deg=48, max_it=400, link_prec=prec, window=window,
                   smear_kind=kind, smear_p1=p1, smear_iters=iters, smear_compat=1)
    if window == gpu.WINDOW_MLP:
        from laph_eigsys_b200 import window as lw
        lw.set_model(s, lw.load_model())
    s.set_links(0, U)
    st, res = s.run()
    assert st == 0, res
    (ev, V, _), ritz = s.get(0), s.ritz(0)
    s.close()
    orc.set_threads(os.cpu_count() or 1)
    Us = orc.smear_ape(U, L, p1, iters, 1) if case == "c4_32" else orc.smear_stout(U, L, p1, iters, 1)
    st, _, Vk, nconv, _, _ = orc.eps_solve(Us, L, 12.0, float(1.1 * (-ev)[-1]), 12, nev, tol=1e-10, max_it=400)
    assert st == 0 and nconv >= nev
    Vo, _ = orc.fix_phase(Vk)
    r = _check(orc, Us, L, V, Vo, ritz[nev], 1e-9, False, f"{case} vs Krylov-Schur")
    # Davis-Kahan: sin of the largest angle <= residual / gap after lambda_nev (the solver's own Ritz value nev + 1)
    gap = float(ritz[nev] - (-ev)[-1])
    assert gap > 0
    assert r["block_proj"] <= max(10 * 1e-9 * 12.0 / gap, 1e-8), (r["block_proj"], gap)


def test_largest_lattice_in_the_suite_64(gpu, orc):
    """64^3 (262144 sites, vectors of 786432 complex entries: past every 32-bit product of sites and columns the
    smaller cases reach), stout 2 x 0.1: the MatShell product T_12(B) x against the oracle's tv_iter (1e-13; the
    fused product's grid-stride form, more CTAs than co-resident slots), and the block solver's nev = 16 against the
    oracle's Krylov-Schur (eigenvalues to 1e-10, residuals at the tolerance)."""
    L, nev, tol = 64, 16, 1e-9
    U = _links(gpu, L, 1, 0.3, 1240, [0])[0]
    orc.set_threads(os.cpu_count() or 1)
    Us = orc.smear_stout(U, L, 0.1, 2, 1)
    ctx = gpu.Context(L, 12.0, 0.6, 12)
    ctx.set_links(Us)
    rng = np.random.default_rng(7)
    x = rng.normal(size=3 * L ** 3) + 1j * rng.normal(size=3 * L ** 3)
    y = ctx.matmult(x, 12)
    ctx.close()
    yr = orc.tv_iter(Us, L, 12.0, 0.6, 12, x)
    assert np.linalg.norm(y - yr) / np.linalg.norm(yr) <= 1e-13
    out = _solve(gpu, L, nev, [U], tol, 48, smear_kind=gpu.SMEAR_STOUT, smear_p1=0.1, smear_iters=2, smear_compat=1)
    (ev, V, _), ritz = out[0]
    st, _, Vk, nconv, _, _ = orc.eps_solve(Us, L, 12.0, float(1.5 * (-ev)[-1]), 12, nev, tol=1e-10, max_it=400)
    assert st == 0 and nconv >= nev
    Vo, _ = orc.fix_phase(Vk)
    _check(orc, Us, L, V, Vo, ritz[nev], tol, False, "64^3 vs Krylov-Schur")
