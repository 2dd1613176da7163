"""laph_tune_hyp (the tune_hyp replacement): one batched solve over the
(alpha_1, alpha_2) grid of HYP parameters for one timeslice; lowest
eigenvalues and files against the oracle (HYP smearing + dense eigh)."""
import os
import subprocess

import numpy as np
import pytest

import laph_eigsys_b200 as lb

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "laph_eigsys_b200", "laph_tune_hyp")


def reference_grid(a1i, a1f, a2i, a2f):
    """The reference's loops: for (a = a_i; a <= a_f; a += 0.05), in double precision."""
    out = []
    a1 = a1i
    while a1 <= a1f:
        a2 = a2i
        while a2 <= a2f:
            out.append((a1, a2))
            a2 += 0.05
        a1 += 0.05
    return out


def test_tune_hyp_cli(gpu, orc, tmp_path):
    L, T, nev, cfgno, ts, it = 6, 3, 8, 1229, 1, 2
    conf = lb.gauge_random(L, T, 0.4, 1229)
    gdir = tmp_path / "gauges"
    gdir.mkdir()
    lb.lime_write_gauge(gdir / f"conf.{cfgno:04d}", conf, L, T)
    out = tmp_path / "out"
    out.mkdir()
    (tmp_path / "parameters.txt").write_text(
        f"config_path = {gdir}\nresult_path = {out}\nLT = {T}\nLX = {L}\nNEV = {nev}\niter = {it}\n"
        f"alpha_1_i = 0.55\nalpha_1_f = 0.65\nalpha_2_i = 0.45\nalpha_2_f = 0.5\ntol = 1e-11\n")
    r = subprocess.run([EXE, "--ts", str(ts), str(cfgno)], cwd=tmp_path, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    grid = reference_grid(0.55, 0.65, 0.45, 0.5)
    table = r.stdout.split("#alpha1\talpha2\tlowest_ev\n")[1].strip().splitlines()
    assert len(table) == len(grid)
    U = lb.spatial_links(conf[ts])
    for (a1, a2), row in zip(grid, table):
        Us = orc.smear_hyp(U, L, a1, a2, it)
        w = np.linalg.eigvalsh(orc.neglap_dense(Us, L))
        low = float(row.split("\t")[2])
        assert abs(low + w[0]) < 1e-9, (a1, a2)
        ev = lb.read_eigenvalues_bin(out, f"eigenvalues_hyp-{it}_a1-{a1:.2f}_a2-{a2:.2f}", cfgno, ts, nev)
        assert np.abs(np.sort(-ev) - w[:nev]).max() < 1e-9
        ph = lb.read_eigenvalues_bin(out, f"phases_hyp-{it}_a1-{a1:.2f}_a2-{a2:.2f}", cfgno, ts, nev)
        assert ph.shape == (nev,)


def test_per_problem_smearing_matches_separate_solves(gpu, orc):
    """Copies of one timeslice with their own APE alpha in one batch equal the oracle per alpha."""
    L, nev = 6, 10
    U = lb.spatial_links(lb.gauge_random(L, 1, 0.4, 31)[0])
    alphas = [0.3, 0.5, 0.7]
    s = gpu.Solver([(L, nev)] * 3, tol=1e-10, deg=8, max_it=300, smear_kind=gpu.SMEAR_APE, smear_p1=0.5,
                   smear_iters=2, smear_compat=1)
    for i, a in enumerate(alphas):
        s.set_links(i, U)
        s.set_smear(i, a)
    st, _ = s.run()
    assert st == 0
    for i, a in enumerate(alphas):
        w = np.linalg.eigvalsh(orc.neglap_dense(orc.smear_ape(U, L, a, 2, 1), L))
        ev, _, _ = s.get(i, vectors=False)
        assert np.abs(-ev - w[:nev]).max() < 1e-9
    s.close()
