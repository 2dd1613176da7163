"""The whole solve as one graph launch (the default): its WHILE node repeats the
outer iteration on the device, SWITCH nodes pick each pass's filter steps, and
small kernels make the decisions the host loop makes between its graph
launches (degree cap, the learned window's check, convergence).  Both loops
must run the same kernels in the same order, so they give the same iterations
and bitwise the same eigenpairs; an uneven batch (timeslices of different L
and nev in one launch) is checked against the oracle's FP64 Krylov-Schur (the
reference's EPSSolve on T_12(B), src/ev_ts.cpp:231-263) at 16^3 and 24^3."""
import os

import numpy as np
import pytest

from conftest import random_links

pytestmark = pytest.mark.gpu


def _solve(gpu, probs, links, **kw):
    s = gpu.Solver(probs, **kw)
    if kw.get("window") == gpu.WINDOW_MLP:
        from laph_eigsys_b200 import window
        window.set_model(s, window.load_model())
    for i, U in enumerate(links):
        s.set_links(i, U)
    st, res = s.run()
    out = dict(status=st, res=res, eig=[s.get(i) for i in range(len(probs))], counters=s.counters(),
               fbytes=s.filter_bytes(), timings=s.timings(), loop=s.loop_info())
    s.close()
    return out


@pytest.mark.parametrize("window", ["lanczos", "mlp"])
def test_device_loop_matches_host_loop(gpu, window):
    probs = [(8, 20), (6, 12), (10, 30), (8, 20)]
    links = [random_links(L, 0.35, 3100 + i) for i, (L, _) in enumerate(probs)]
    kw = dict(smear_kind=gpu.SMEAR_STOUT, smear_p1=0.1, smear_iters=3, guard=16, tol=1e-10, deg=24, max_it=200,
              window=gpu.WINDOW_MLP if window == "mlp" else gpu.WINDOW_LANCZOS)
    dev = _solve(gpu, probs, links, host_loop=0, **kw)
    host = _solve(gpu, probs, links, host_loop=1, **kw)
    assert dev["status"] == 0 and host["status"] == 0
    assert dev["loop"] == (1, 1), dev["loop"]  # the whole solve was one graph launch
    assert host["loop"][0] == 0 and host["loop"][1] >= 2
    for a, b in zip(dev["res"], host["res"]):
        assert a["iters"] == b["iters"] and a["nconv"] == b["nconv"]
        assert a["window_fallback"] == b["window_fallback"]
        assert a["lam_max"] == b["lam_max"]
    for (ea, va, pa), (eb, vb, pb) in zip(dev["eig"], host["eig"]):
        assert np.array_equal(ea, eb)
        assert np.array_equal(va, vb)
        assert np.array_equal(pa, pb)
    assert dev["counters"][:2] == host["counters"][:2]
    assert np.allclose(dev["fbytes"], host["fbytes"], rtol=1e-12)
    t = dev["timings"]
    assert t[1] > 0 and t[3] >= t[1] and t[0] > 0


def test_device_loop_reports_not_converged_at_max_it(gpu):
    L, nev = 8, 30
    s = gpu.Solver([(L, nev)], guard=16, tol=1e-13, deg=8, max_it=3)
    s.set_links(0, random_links(L, 0.4, 3200))
    st, res = s.run()
    assert st == gpu._lib.LAPH_ENOTCONV
    assert res[0]["status"] == gpu._lib.LAPH_ENOTCONV and res[0]["iters"] <= 3
    s.close()


def test_uneven_batch_in_one_launch_matches_oracle_krylov_schur(gpu, orc):
    """16^3 (nev 60) and 24^3 (nev 120) timeslices, APE 0.5 x 10 as the mixed-volume benchmark configuration, in one
    batch and one graph launch, each against the oracle's smearing + FP64 Krylov-Schur on T_12(B): eigenvalues
    (Rayleigh quotients) to 1e-10 relative each, residuals at the tolerance, tr(V^dag V) = nev, and the nev-block
    subspace to the residual over the gap.  The oracle's Krylov-Schur runs at 1e-10 relative to |theta| (near the
    window's edge theta is close to 1 and a tighter test needs hundreds of restarts on these smooth fields)."""
    specs = [(16, 60, 1230, 0), (24, 120, 1231, 0), (16, 60, 1230, 1)]
    links, probs = [], []
    for L, nev, seed, t in specs:
        conf = gpu.gauge_random(L, t + 1, 0.3, seed)
        links.append(np.ascontiguousarray(conf[t, :, 1:4]))
        probs.append((L, nev))
    tol = 1e-11
    out = _solve(gpu, probs, links, smear_kind=gpu.SMEAR_APE, smear_p1=0.5, smear_iters=10, smear_compat=1,
                 guard=16, tol=tol, deg=48, max_it=300, window=gpu.WINDOW_LANCZOS)
    assert out["status"] == 0
    orc.set_threads(os.cpu_count() or 1)
    for (L, nev), U, (ev, V, _) in zip(probs, links, out["eig"]):
        Us = orc.smear_ape(U, L, 0.5, 10, 1)
        lam = -ev
        st, _, Vk, _, _, _ = orc.eps_solve(Us, L, 12.0, float(1.1 * lam[-1]), 12, nev, tol=1e-10, max_it=400)
        assert st == 0
        Vo, _ = orc.fix_phase(Vk)
        r = orc.compare_eigensystems(Us, L, V, Vo)
        print(L, nev, {k: r[k] for k in ("max_rel_eig", "max_resid_checked", "max_resid_oracle", "block_proj",
                                           "max_vec_phase_fixed", "gap_min_isolated")})
        assert r["max_rel_eig"] <= 1e-10
        assert r["max_resid_checked"] <= tol * 1.01
        assert abs(r["trace_vdv_checked"] - nev) <= 1e-9
        # both blocks span the lowest nev eigenvectors to within their residuals over the gap after lambda_nev
        assert r["block_proj"] <= 1e-6


def test_async_read_back_overlaps_the_next_run(gpu):
    """laph_solver_get_async queues each problem's results on the solver's read-back stream; the next run may start
    at once (it waits only for the conversions out of the block) and the first run's results still land intact in
    the host buffers, equal to what laph_solver_get returned for that run."""
    import torch
    probs = [(8, 20), (10, 30), (6, 12)]
    s = gpu.Solver(probs, smear_kind=gpu.SMEAR_STOUT, smear_p1=0.1, smear_iters=2, guard=16, tol=1e-10, deg=24)
    sets = [[random_links(L, 0.35, 3300 + 10 * k + i) for i, (L, _) in enumerate(probs)] for k in range(2)]
    ref = []
    for k in range(2):  # reference results of each link set, read synchronously
        for i, U in enumerate(sets[k]):
            s.set_links(i, U)
        assert s.run()[0] == 0
        ref.append([s.get(i) for i in range(len(probs))])
    bufs = [[(torch.empty(nev, dtype=torch.float64, pin_memory=True).numpy(),
              torch.empty((3 * L ** 3) * nev, dtype=torch.complex128, pin_memory=True).numpy(),
              torch.empty(nev, dtype=torch.float64, pin_memory=True).numpy()) for L, nev in probs] for _ in range(2)]
    for k in range(2):
        for i, U in enumerate(sets[k]):
            s.set_links(i, U)
        assert s.run()[0] == 0
        for i in range(len(probs)):
            s.get_async(i, *bufs[k][i])
    s.wait()
    for k in range(2):
        for i, (L, nev) in enumerate(probs):
            ev, V, ph = ref[k][i]
            e, v, p = bufs[k][i]
            assert np.array_equal(e, ev) and np.array_equal(p, ph)
            assert np.array_equal(v.reshape(nev, 3 * L ** 3).T, V)
    s.close()


@pytest.mark.parametrize("prec", ["fp32", "bf16"])
def test_filter_tiles_are_bitwise_identical(gpu, prec):
    """The filter's site tile (64, 128 or 256 sites per CTA, an autotuner axis) changes only which CTA computes a
    site, not the arithmetic: every tile gives bitwise the same eigenpairs, on a batch with a ragged last tile
    (10^3 = 1000 sites, 12^3 = 1728).  The same holds for where the backward links wait between columns (shared
    memory, filter_kernel 1, or tensor memory, filter_kernel 2) and for where a thread's operands wait (registers,
    or its own slots of a cp.async double buffer, filter_kernel 5): all run the same FMAs in the same order."""
    probs = [(10, 24), (12, 30)]
    links = [random_links(L, 0.35, 3400 + i) for i, (L, _) in enumerate(probs)]
    outs = []
    for variant in (1, 2, 5):
        for tile in (64, 128, 256):
            o = _solve(gpu, probs, links, guard=16, tol=1e-10, deg=24, filter_tile=tile, filter_kernel=variant,
                       link_prec=gpu.LINKS_BF16 if prec == "bf16" else gpu.LINKS_FP32)
            assert o["status"] == 0
            outs.append(o)
    for o in outs[1:]:
        for (ea, va, _), (eb, vb, _) in zip(outs[0]["eig"], o["eig"]):
            assert np.array_equal(ea, eb) and np.array_equal(va, vb)


@pytest.mark.parametrize("prec", ["fp32", "bf16"])
def test_staged_filter_is_bitwise_identical(gpu, prec):
    """filter_kernel 3 feeds the same column loop from a bulk-copy pipeline (X with its x- and y-neighbour rows, S
    and Z staged in shared memory) instead of global loads: the same FMAs in the same order, so the eigenpairs match
    filter_kernel 1 bit for bit.  The batch mixes 16^3 and 32^3 timeslices (two tile geometries in one launch, the
    ring sized for L = 32); a batch with a lattice the staged tiles do not fit (12^3) runs variant 1 instead.
    filter_kernel 4 (the same loop as variant 2 on 512-site bricks of TX planes x 4 z-rows) must match as well."""
    lp = gpu.LINKS_BF16 if prec == "bf16" else gpu.LINKS_FP32
    for probs in ([(16, 40), (32, 24), (16, 20)], [(12, 30), (16, 24)]):
        links = [random_links(L, 0.35, 3500 + i) for i, (L, _) in enumerate(probs)]
        outs = [_solve(gpu, probs, links, guard=16, tol=1e-10, deg=24, filter_kernel=v, link_prec=lp)
                for v in (1, 3, 4)]
        for o in outs:
            assert o["status"] == 0
        for o in outs[1:]:
            for (ea, va, pa), (eb, vb, pb) in zip(outs[0]["eig"], o["eig"]):
                assert np.array_equal(ea, eb) and np.array_equal(va, vb) and np.array_equal(pa, pb)
            assert outs[0]["res"][0]["iters"] == o["res"][0]["iters"]


def test_direct_passes_converge_to_the_same_eigensystem(gpu):
    """Passes whose largest wanted residual is above direct_resid filter V itself in FP32 (T_{m-1}(B) V, no S);
    the correction form takes over below it.  The eigenpairs match a solve without direct passes (eigenvalues to
    1e-10 of lambda_max, the nev-block projectors to the residual over the gap), with the default threshold and
    with direct_resid = 0 (direct until a pass fails to halve the residual, then the correction form: the guard
    that keeps a solve from stalling at the FP32 filter's floor).  BF16 links never take direct passes: their
    results equal the direct_resid = -1 run bit for bit.  Both loops stay bitwise identical with direct passes."""
    probs = [(10, 24), (12, 30)]
    links = [random_links(L, 0.35, 3600 + i) for i, (L, _) in enumerate(probs)]
    kw = dict(smear_kind=gpu.SMEAR_STOUT, smear_p1=0.1, smear_iters=2, guard=16, tol=1e-11, deg=32, max_it=300)
    off = _solve(gpu, probs, links, direct_resid=-1.0, **kw)
    assert off["status"] == 0
    for dr in (1e-3, 0.0):
        on = _solve(gpu, probs, links, direct_resid=dr, **kw)
        assert on["status"] == 0, dr
        for (ea, va, _), (eb, vb, _) in zip(on["eig"], off["eig"]):
            assert np.max(np.abs(ea - eb)) <= 1e-10 * 12.0, dr
            proj = va @ (va.conj().T @ vb) - vb
            assert np.linalg.norm(proj) / np.sqrt(vb.shape[1]) <= 1e-6, dr
    host = _solve(gpu, probs, links, direct_resid=1e-3, host_loop=1, **kw)
    dev = _solve(gpu, probs, links, direct_resid=1e-3, **kw)
    for (ea, va, _), (eb, vb, _) in zip(dev["eig"], host["eig"]):
        assert np.array_equal(ea, eb) and np.array_equal(va, vb)
    assert np.allclose(dev["fbytes"], host["fbytes"], rtol=1e-12)
    bf = [_solve(gpu, probs, links, direct_resid=dr, link_prec=gpu.LINKS_BF16, **kw) for dr in (1e-3, -1.0)]
    for (ea, va, _), (eb, vb, _) in zip(bf[0]["eig"], bf[1]["eig"]):
        assert np.array_equal(ea, eb) and np.array_equal(va, vb)
