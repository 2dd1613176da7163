"""The command-line programs' host logic without a device: argument and
parameters.txt errors, unreadable gauge files, --resume over complete outputs
(which needs no solve), the per-rank timeslice split of the resume list, and
that a solve without a CUDA device stops with an error instead of falling back
to the host."""
import os
import subprocess

import numpy as np
import pytest

import laph_eigsys_b200 as lb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EV_TS = os.path.join(ROOT, "laph_eigsys_b200", "laph_ev_ts")
TUNE = os.path.join(ROOT, "laph_eigsys_b200", "laph_tune_hyp")


# rank / size / device variables of the launchers laph_ev_ts understands
LAUNCHER_VARS = ("LAPH_RANK", "LAPH_WORLD_SIZE", "LAPH_DEVICE", "RANK", "WORLD_SIZE", "LOCAL_RANK",
                 "OMPI_COMM_WORLD_RANK", "OMPI_COMM_WORLD_SIZE", "OMPI_COMM_WORLD_LOCAL_RANK", "PMI_RANK", "PMI_SIZE",
                 "MPI_LOCALRANKID", "SLURM_PROCID", "SLURM_NTASKS", "SLURM_LOCALID", "SLURM_STEP_ID",
                 "SLURM_STEP_NUM_TASKS")


def _run(exe, args, cwd, env=None):
    e = dict(os.environ)
    for k in LAUNCHER_VARS:
        e.pop(k, None)
    e.update(env or {})
    return subprocess.run([exe] + args, cwd=cwd, capture_output=True, text=True, timeout=120, env=e)


def _has_device():
    import torch
    return torch.cuda.is_available()


def _setup(tmp_path, L=4, T=5, nev=6, cfgno=1227, solver="block", extra=""):
    gdir = tmp_path / "gauges"
    gdir.mkdir(exist_ok=True)
    out = tmp_path / "out"
    out.mkdir(exist_ok=True)
    conf = lb.gauge_random(L, T, 0.3, cfgno)
    lb.lime_write_gauge(gdir / f"conf.{cfgno:04d}", conf, L, T)
    (tmp_path / "parameters.txt").write_text(
        f"config_path = {gdir}\nresult_path = {out}\nLT = {T}\nLX = {L}\nNEV = {nev}\n"
        f"alpha_1 = 0.62\nalpha_2 = 0.52\niter = 1\nLAM_L = 12.0\nLAM_C = 1.0\nDEG = 8\nOMP_THRDS = 1\n"
        f"solver = {solver}\nwindow = lanczos\n{extra}")
    return out


def _write_complete_outputs(out, cfgno, t, dim, nev, seed):
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.normal(size=(dim, nev)) + 1j * rng.normal(size=(dim, nev)))
    lb.write_eigsys_bin(out, "eigenvectors", cfgno, t, np.asfortranarray(Q))
    lb.write_eigenvalues_bin(out, "eigenvalues", cfgno, t, -np.linspace(0.1, 1.0, nev))
    lb.write_eigenvalues_bin(out, "phases", cfgno, t, np.zeros(nev))


def test_ev_ts_argument_errors(tmp_path):
    r = _run(EV_TS, [], tmp_path)
    assert r.returncode == 2 and "No configuration number specified!" in r.stdout and "usage" in r.stderr
    r = _run(EV_TS, ["--conf", "1", "--bogus"], tmp_path)
    assert r.returncode == 2 and "usage" in r.stderr
    r = _run(EV_TS, ["--help"], tmp_path)
    assert r.returncode == 1 and "usage" in r.stderr
    r = _run(EV_TS, ["--conf", "1"], tmp_path)  # no parameters.txt in the working directory
    assert r.returncode == 1 and "parameters" in r.stderr


def test_ev_ts_missing_or_damaged_gauge(tmp_path):
    _setup(tmp_path)
    r = _run(EV_TS, ["--conf", "99"], tmp_path)  # conf.0099 does not exist
    assert r.returncode == 1 and "read gauge" in r.stderr
    # a file whose binary record has the wrong size for LT x LX^3
    bad = tmp_path / "gauges" / "conf.0098"
    lb.lime_write_gauge(bad, lb.gauge_random(4, 3, 0.3, 1), 4, 3)
    r = _run(EV_TS, ["--conf=98"], tmp_path)
    assert r.returncode == 1 and "read gauge" in r.stderr


def test_ev_ts_resume_over_complete_outputs_needs_no_solve(tmp_path):
    L, T, nev, cfgno = 4, 5, 6, 1227
    out = _setup(tmp_path, L, T, nev, cfgno)
    for t in range(T):
        _write_complete_outputs(out, cfgno, t, 3 * L ** 3, nev, t)
    before = {p.name: p.read_bytes() for p in out.iterdir()}
    r = _run(EV_TS, ["--conf", str(cfgno), "--resume"], tmp_path)
    assert r.returncode == 0, r.stderr
    skipped = [ln for ln in r.stdout.splitlines() if '"skipped"' in ln]
    assert [int(ln.split(":")[1].split(",")[0]) for ln in skipped] == list(range(T))
    assert {p.name: p.read_bytes() for p in out.iterdir()} == before
    # the reference's MPI split: rank 1 of 2 owns timeslices 3, 4 (rank 0 takes the extra one), whichever
    # launcher sets the rank and size
    for env in ({"LAPH_WORLD_SIZE": "2", "LAPH_RANK": "1"}, {"WORLD_SIZE": "2", "RANK": "1"},
                {"OMPI_COMM_WORLD_SIZE": "2", "OMPI_COMM_WORLD_RANK": "1"}, {"PMI_SIZE": "2", "PMI_RANK": "1"},
                {"SLURM_STEP_ID": "0", "SLURM_STEP_NUM_TASKS": "2", "SLURM_PROCID": "1"}):
        r = _run(EV_TS, ["--conf", str(cfgno), "--resume"], tmp_path, env)
        assert r.returncode == 0, r.stderr
        assert [ln for ln in r.stdout.splitlines() if '"skipped"' in ln] == skipped[3:], env
    # rank 0 of 3 under srun: timeslices 0, 1
    r = _run(EV_TS, ["--conf", str(cfgno), "--resume"], tmp_path,
             {"SLURM_STEP_ID": "0", "SLURM_STEP_NUM_TASKS": "3", "SLURM_PROCID": "0", "SLURM_NTASKS": "8"})
    assert [ln for ln in r.stdout.splitlines() if '"skipped"' in ln] == skipped[:2]
    assert '"launcher": "srun", "rank": 0, "size": 3' in r.stdout


def test_ev_ts_plain_process_in_a_slurm_allocation_takes_every_timeslice(tmp_path):
    """A process started inside an sbatch allocation of 8 tasks, but not by srun, sees SLURM_NTASKS = 8 and
    SLURM_PROCID = 0; those describe the allocation, so laph_ev_ts must run as rank 0 of 1 and take all
    timeslices.  Rank and size never mix launchers either (torchrun's rank with Slurm's size)."""
    L, T, nev, cfgno = 4, 5, 6, 1227
    out = _setup(tmp_path, L, T, nev, cfgno)
    for t in range(T):
        _write_complete_outputs(out, cfgno, t, 3 * L ** 3, nev, t)
    for env in ({"SLURM_NTASKS": "8", "SLURM_PROCID": "0", "SLURM_LOCALID": "0"},
                {"SLURM_NTASKS": "8", "SLURM_PROCID": "0", "RANK": "3"}):
        r = _run(EV_TS, ["--conf", str(cfgno), "--resume"], tmp_path, env)
        assert r.returncode == 0, r.stderr
        assert '"launcher": "none", "rank": 0, "size": 1, "device": 0, "t0": 0, "t1": 4' in r.stdout, (env, r.stdout)
        assert len([ln for ln in r.stdout.splitlines() if '"skipped"' in ln]) == T


@pytest.mark.parametrize("damage", ["short_phases", "bad_trace", "missing_eigenvalues"])
def test_ev_ts_resume_detects_incomplete_outputs(tmp_path, damage):
    """An incomplete timeslice is not skipped; without a device the solve that follows stops with an error."""
    L, T, nev, cfgno = 4, 3, 6, 1229
    out = _setup(tmp_path, L, T, nev, cfgno)
    dim = 3 * L ** 3
    for t in range(T):
        _write_complete_outputs(out, cfgno, t, dim, nev, 10 + t)
    if damage == "short_phases":
        (out / f"phases.{cfgno:04d}.001").write_bytes(b"\0" * 8)
    elif damage == "bad_trace":
        raw = np.fromfile(out / f"eigenvectors.{cfgno:04d}.001", dtype=np.complex128) * 1.01
        raw.tofile(out / f"eigenvectors.{cfgno:04d}.001")
    else:
        os.remove(out / f"eigenvalues.{cfgno:04d}.001")
    if _has_device():
        pytest.skip("a device is present: the solve would run (covered by the GPU command-line tests)")
    r = _run(EV_TS, ["--conf", str(cfgno), "--resume"], tmp_path)
    skipped = [int(ln.split(":")[1].split(",")[0]) for ln in r.stdout.splitlines() if '"skipped"' in ln]
    assert skipped == [0, 2]
    assert r.returncode == 1 and "laph_ev_ts: device memory:" in r.stderr


def test_ev_ts_without_device_fails_loudly(tmp_path):
    if _has_device():
        pytest.skip("a device is present")
    for solver, extra, stage in (("block", "", "device memory"), ("plain", "", "context"),
                                 ("block", "autotune = 2\n", "autotune")):
        _setup(tmp_path, solver=solver, extra=extra)
        r = _run(EV_TS, ["--conf", "1227"], tmp_path)
        assert r.returncode == 1 and f"laph_ev_ts: {stage}:" in r.stderr, (solver, r.stderr)
        assert not any(p.name.startswith("eigen") for p in (tmp_path / "out").iterdir())


def test_tune_hyp_argument_and_grid_errors(tmp_path):
    r = _run(TUNE, [], tmp_path)
    assert r.returncode == 2 and "usage" in r.stderr
    r = _run(TUNE, ["--bogus", "x", "3"], tmp_path)
    assert r.returncode == 2 and "usage" in r.stderr
    r = _run(TUNE, ["3"], tmp_path)
    assert r.returncode == 1 and "parameters" in r.stderr
    _setup(tmp_path, extra="alpha_1_i = 0.4\nalpha_1_f = 0.5\nalpha_2_i = 0.3\nalpha_2_f = 0.35\n")
    r = _run(TUNE, ["1227"], tmp_path)  # the reference's timeslice 10 is outside LT = 5
    assert r.returncode == 2 and "outside 0..4" in r.stderr
    r = _run(TUNE, ["--ts", "2", "1226"], tmp_path)
    assert r.returncode == 1 and "read gauge" in r.stderr
    (tmp_path / "parameters.txt").write_text((tmp_path / "parameters.txt").read_text() + "alpha_1_f = 0.3\n")
    r = _run(TUNE, ["--ts", "2", "1227"], tmp_path)  # alpha_1_f < alpha_1_i: no grid point
    assert r.returncode == 2 and "empty" in r.stderr
    if not _has_device():
        (tmp_path / "parameters.txt").write_text((tmp_path / "parameters.txt").read_text() + "alpha_1_f = 0.5\n")
        r = _run(TUNE, ["--ts", "2", "--conf", "1227"], tmp_path)
        assert r.returncode == 1 and "laph_tune_hyp: device memory:" in r.stderr


SHAPE = os.path.join(ROOT, "laph_eigsys_b200", "laph_sourceshape")


def _shape_setup(tmp_path, L=6, nev=8, cfgno=1227, t=3):
    ind = tmp_path / "eigsys"
    ind.mkdir(exist_ok=True)
    (tmp_path / "parameters.txt").write_text(f"in_path = {ind}\nLT = 8\nLX = {L}\nNEV = {nev}\n")
    rng = np.random.default_rng(cfgno + t)
    dim = 3 * L ** 3
    Q, _ = np.linalg.qr(rng.normal(size=(dim, nev)) + 1j * rng.normal(size=(dim, nev)))
    Q = np.asfortranarray(Q)
    lb.write_eigsys_bin(ind, "eigenvectors", cfgno, t, Q)
    return ind, Q


def test_sourceshape_cli_errors(tmp_path):
    r = _run(SHAPE, [], tmp_path)
    assert r.returncode == 2 and "configuration timeslice dim(V)" in r.stdout
    r = _run(SHAPE, ["1", "2"], tmp_path)
    assert r.returncode == 2
    r = _run(SHAPE, ["--bogus", "1", "2", "3"], tmp_path)
    assert r.returncode == 2 and "usage" in r.stderr
    r = _run(SHAPE, ["1227", "3", "8"], tmp_path)
    assert r.returncode == 1 and "parameters" in r.stderr
    ind, Q = _shape_setup(tmp_path)
    r = _run(SHAPE, ["1227", "4", "8"], tmp_path)  # no eigensystem for timeslice 4
    assert r.returncode == 1 and "read eigenvectors" in r.stderr
    r = _run(SHAPE, ["1227", "3", "9"], tmp_path)  # more columns than the file holds
    assert r.returncode == 1 and "read eigenvectors" in r.stderr
    r = _run(SHAPE, ["--weighted", "1227", "3", "8"], tmp_path)  # no eigenvalues file
    assert r.returncode == 1 and "read eigenvalues" in r.stderr
    (Q * 1.01).tofile(ind / "eigenvectors.1227.003")  # fails check_trace
    r = _run(SHAPE, ["1227", "3", "8"], tmp_path)
    assert r.returncode == 1 and "damaged" in r.stderr
    if not _has_device():
        _shape_setup(tmp_path)
        r = _run(SHAPE, ["1227", "3", "8"], tmp_path)
        assert r.returncode == 1 and "laph_sourceshape: sourceshape:" in r.stderr
        assert not list(tmp_path.glob("sourceshape_nev*"))


def test_window_model_file_and_ev_ts_loading(tmp_path):
    """The shipped learned-window model (data/window_mlp.bin: "LAPHMLP1", int32 nparams, int32 nnorm, float32
    values, then the training record as JSON) has the shape the library expects and finite values; laph_ev_ts with
    window = mlp loads it (from beside the executable) and, without a device, stops at its first device step, not
    at the model."""
    import json
    from laph_eigsys_b200 import window as lw
    raw = open(lw.MODEL_PATH, "rb").read()
    assert raw[:8] == b"LAPHMLP1"
    npar, nnorm = (int(v) for v in np.frombuffer(raw[8:16], dtype="<i4"))
    end = 16 + 4 * (npar + nnorm)
    assert npar == lb.lib.laph_mlp_nparams() and len(raw) >= end
    meta = json.loads(raw[end:].decode()) if len(raw) > end else {}
    assert "val_cut_rel_err_median" in meta
    m = lw.load_model()
    assert m.size == npar + nnorm and np.all(np.isfinite(m))
    if _has_device():
        pytest.skip("a device is present")
    _setup(tmp_path, extra="window = mlp\n")
    r = _run(EV_TS, ["--conf", "1227"], tmp_path)
    assert r.returncode == 1 and "laph_ev_ts: device memory:" in r.stderr and "window" not in r.stderr
