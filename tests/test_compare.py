"""python -m laph_eigsys_b200.compare on CPU: two eigensystem directories that differ only by column phases and
a rotation inside a degenerate cluster compare equal (projector distance and eigenvalue difference at rounding);
a block with a column from outside the subspace does not."""
import json
import subprocess
import sys

import numpy as np

import laph_eigsys_b200 as lb
from laph_eigsys_b200.compare import cluster_ends, compare_timeslice

ROOT = __import__("os").path.dirname(__import__("os").path.dirname(__import__("os").path.abspath(__file__)))


def _system(seed, L=3, nev=6):
    rng = np.random.default_rng(seed)
    dim = 3 * L ** 3
    Q, _ = np.linalg.qr(rng.normal(size=(dim, dim)) + 1j * rng.normal(size=(dim, dim)))
    lam = np.array([0.0, 0.0, 0.0, 0.5, 0.5, 1.0, 1.2, 1.5])  # clusters {0,1,2}, {3,4}, {5}; nev = 6 closes {5}
    return Q[:, :nev], -lam[:nev], Q, lam


def test_cluster_ends():
    lam = np.array([0.0, 0.0, 0.0, 0.5, 0.5, 1.0, 1.0, 2.0])
    assert cluster_ends(lam, 6, 1e-6) == [3, 5]          # the {1.0, 1.0} cluster is cut by nev = 6
    assert cluster_ends(lam, 7, 1e-6) == [3, 5, 7]
    assert cluster_ends(lam[:6], 6, 1e-6) == [3, 5, 6]   # nothing known beyond nev: the last cluster counts


def test_compare_equal_up_to_phases_and_cluster_rotation(tmp_path):
    U, ev, Q, lam = _system(1)
    rng = np.random.default_rng(2)
    R, _ = np.linalg.qr(rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3)))
    V = U.copy()
    V[:, :3] = V[:, :3] @ R                                   # another basis of the 3-fold cluster
    V = V * np.exp(1j * rng.uniform(-np.pi, np.pi, 6))[None, :]  # column phases
    r = compare_timeslice(U, V, ev, ev)
    assert r["proj"] < 1e-12 and r["dlam"] == 0.0 and r["clusters_checked"] == 3
    assert r["col"] > 0.1                                     # column 5 (simple) carries a different phase in V
    Uf, _ = lb.fix_phase(U)
    Vf, _ = lb.fix_phase(V)
    r = compare_timeslice(Uf, Vf, ev, ev)
    assert r["col"] < 1e-14 and r["phase"] < 1e-14            # phase-fixed: the simple column agrees
    W = U.copy()
    W[:, 5] = Q[:, 7]                                         # a vector of another eigenvalue
    r = compare_timeslice(U, W, ev, ev)
    assert r["proj"] > 0.99
    # through the files and the command line
    for name, blk in (("a", U), ("b", V), ("c", W)):
        d = tmp_path / name
        d.mkdir()
        lb.write_eigsys_bin(d, "eigenvectors", 1227, 2, np.asfortranarray(blk))
        lb.write_eigenvalues_bin(d, "eigenvalues", 1227, 2, ev)
    run = lambda x, y: subprocess.run(  # noqa: E731
        [sys.executable, "-m", "laph_eigsys_b200.compare", str(tmp_path / x), str(tmp_path / y), "--conf", "1227",
         "--lx", "3", "--nev", "6", "--timeslices", "2", "--eigenvalues", "--json"],
        cwd=ROOT, capture_output=True, text=True, timeout=120)
    r = run("a", "b")
    assert r.returncode == 0, r.stderr
    worst = json.loads(r.stdout.splitlines()[-1])["worst"]
    assert worst["proj"] < 1e-12 and worst["dlam"] == 0.0
    worst = json.loads(run("a", "c").stdout.splitlines()[-1])["worst"]
    assert worst["proj"] > 0.99
