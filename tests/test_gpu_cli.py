"""laph_ev_ts end to end (the ev_ts replacement): LIME input, parameters.txt,
the reference's output files, for both the plain MatShell + EPS loop and the
batched solver; eigenvalues against the oracle pipeline (HYP smearing + dense
eigendecomposition of -Delta)."""
import os
import subprocess

import numpy as np
import pytest

import laph_eigsys_b200 as lb

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "laph_eigsys_b200", "laph_ev_ts")
# one process, device 0: no launcher's rank, size or device variables reach the programs
ENV = {k: v for k, v in os.environ.items()
       if k not in ("LAPH_RANK", "LAPH_WORLD_SIZE", "LAPH_DEVICE", "RANK", "WORLD_SIZE", "LOCAL_RANK",
                    "OMPI_COMM_WORLD_RANK", "OMPI_COMM_WORLD_SIZE", "OMPI_COMM_WORLD_LOCAL_RANK", "PMI_RANK",
                    "PMI_SIZE", "MPI_LOCALRANKID", "SLURM_PROCID", "SLURM_NTASKS", "SLURM_LOCALID")}


@pytest.mark.parametrize("solver", ["block", "plain"])
def test_ev_ts_cli(gpu, orc, tmp_path, solver):
    L, T, nev, cfgno = 6, 3, 10, 1227
    conf = lb.gauge_random(L, T, 0.4, 1227)
    gdir = tmp_path / "gauges"
    gdir.mkdir()
    lb.lime_write_gauge(gdir / f"conf.{cfgno:04d}", conf, L, T)
    out = tmp_path / "out"
    out.mkdir()
    # LAM_C above lambda_nev of every timeslice
    refs = []
    for t in range(T):
        Us = orc.smear_hyp(lb.spatial_links(conf[t]), L, 0.62, 0.52, 2)
        refs.append(np.linalg.eigvalsh(orc.neglap_dense(Us, L)))
    lam_c = max(0.5 * (r[nev + 2] + r[nev + 3]) for r in refs)
    (tmp_path / "parameters.txt").write_text(
        f"config_path = {gdir}\nresult_path = {out}\nLT = {T}\nLX = {L}\nNEV = {nev}\n"
        f"alpha_1 = 0.62\nalpha_2 = 0.52\niter = 2\nLAM_L = 12.0\nLAM_C = {lam_c}\nDEG = 8\nOMP_THRDS = 2\n"
        f"tol = 1e-11\nsolver = {solver}\n")
    r = subprocess.run([EXE, "--conf", str(cfgno)], cwd=tmp_path, capture_output=True, text=True, timeout=600, env=ENV)
    assert r.returncode == 0, r.stderr
    # one line per timeslice, plus the rank's launcher line
    assert len([ln for ln in r.stdout.splitlines() if ln.startswith('{"t"')]) == T
    assert sum(ln.startswith('{"launcher"') for ln in r.stdout.splitlines()) == 1
    for t in range(T):
        ev = lb.read_eigenvalues_bin(out, "eigenvalues", cfgno, t, nev)
        V = lb.read_eigsys_bin(out, "eigenvectors", cfgno, t, 3 * L ** 3, nev)  # runs check_trace
        ph = lb.read_eigenvalues_bin(out, "phases", cfgno, t, nev)
        tol = 1e-9 if solver == "block" else 1e-6  # recover_spectrum loses digits near theta ~ 1
        assert np.abs(np.sort(-ev) - refs[t][:nev]).max() < tol
        assert np.abs(V[0].imag).max() < 1e-12
        assert ph.shape == (nev,)


def test_ev_ts_cli_fp32_input_and_resume(gpu, orc, tmp_path):
    """Single-precision ILDG input (widened to FP64 on reading) and --resume, which solves only the timeslices
    whose outputs are missing or incomplete."""
    L, T, nev, cfgno = 6, 3, 10, 1228
    conf = lb.gauge_random(L, T, 0.4, 1228)
    gdir = tmp_path / "gauges"
    gdir.mkdir()
    lb.lime_write_gauge(gdir / f"conf.{cfgno:04d}", conf, L, T, precision=32)
    conf32, _ = lb.lime_read_gauge_any(gdir / f"conf.{cfgno:04d}", T, L, 0, T - 1)
    out = tmp_path / "out"
    out.mkdir()
    refs = []
    for t in range(T):
        Us = orc.smear_hyp(lb.spatial_links(conf32[t]), L, 0.62, 0.52, 2)
        refs.append(np.linalg.eigvalsh(orc.neglap_dense(Us, L)))
    (tmp_path / "parameters.txt").write_text(
        f"config_path = {gdir}\nresult_path = {out}\nLT = {T}\nLX = {L}\nNEV = {nev}\n"
        f"alpha_1 = 0.62\nalpha_2 = 0.52\niter = 2\nLAM_L = 12.0\nLAM_C = 1.0\nDEG = 8\nOMP_THRDS = 2\n"
        f"tol = 1e-11\nsolver = block\n")
    r = subprocess.run([EXE, "--conf", str(cfgno)], cwd=tmp_path, capture_output=True, text=True, timeout=600, env=ENV)
    assert r.returncode == 0, r.stderr
    assert "single-precision" in r.stdout
    for t in range(T):
        ev = lb.read_eigenvalues_bin(out, "eigenvalues", cfgno, t, nev)
        assert np.abs(np.sort(-ev) - refs[t][:nev]).max() < 1e-9
    before = lb.read_eigenvalues_bin(out, "eigenvalues", cfgno, 1, nev)
    # damage timeslice 1's phases file; resume must redo exactly that timeslice
    (out / f"phases.{cfgno:04d}.001").write_bytes(b"\0" * 8)
    r = subprocess.run([EXE, "--conf", str(cfgno), "--resume"], cwd=tmp_path, capture_output=True, text=True, env=ENV,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert sum('"skipped"' in ln for ln in lines) == T - 1
    assert sum('"solver": "block"' in ln and '"t": 1,' in ln for ln in lines) == 1
    assert os.path.getsize(out / f"phases.{cfgno:04d}.001") == 8 * nev
    after = lb.read_eigenvalues_bin(out, "eigenvalues", cfgno, 1, nev)
    assert np.abs(after - before).max() < 1e-9


@pytest.mark.parametrize("weighted", [False, True])
def test_sourceshape_cli(gpu, orc, tmp_path, weighted):
    """laph_sourceshape CONFIG T NEV (the reference's sourceshape program) against the oracle's source shape and
    radius average of the same eigensystem file."""
    L, nev, cfgno, t = 6, 8, 1227, 3
    ind = tmp_path / "eigsys"
    ind.mkdir()
    (tmp_path / "parameters.txt").write_text(f"in_path = {ind}\nLT = 8\nLX = {L}\nNEV = {nev}\n")
    rng = np.random.default_rng(5)
    dim = 3 * L ** 3
    Q, _ = np.linalg.qr(rng.normal(size=(dim, nev)) + 1j * rng.normal(size=(dim, nev)))
    Q = np.asfortranarray(Q)
    lb.write_eigsys_bin(ind, "eigenvectors", cfgno, t, Q)
    ev = -np.sort(rng.uniform(0.1, 2.0, nev))
    lb.write_eigenvalues_bin(ind, "eigenvalues", cfgno, t, ev)
    exe = os.path.join(ROOT, "laph_eigsys_b200", "laph_sourceshape")
    args = (["--weighted"] if weighted else []) + [str(cfgno), str(t), str(nev)]
    r = subprocess.run([exe] + args, cwd=tmp_path, capture_output=True, text=True, timeout=300, env=ENV)
    assert r.returncode == 0, r.stderr
    Vw = Q * np.sqrt(np.abs(ev))[None, :] if weighted else Q
    rr, aa = orc.sourceshape_avg(L, orc.sourceshape(Vw, L))
    raw = np.fromfile(tmp_path / f"sourceshape_nev{nev}.{cfgno:04d}.{t:03d}.bin", dtype=np.float64).reshape(-1, 2)
    assert np.array_equal(raw[:, 0], rr)
    assert np.abs(raw[:, 1] - aa).max() <= 1e-12 * np.abs(aa).max()
    txt = open(tmp_path / f"sourceshape_nev{nev}.{cfgno}.{t}").read().splitlines()
    assert txt[0] == "#r\tpsi(r)" and len(txt) == len(rr) + 1
