"""The kernels under the bounds-checked build (liblaph_gpu_check.so, -DLAPH_CHECK)
on small lattices (4^3 to 16^3): the self-test shows an index past its bound
being recorded (and its store redirected in bounds), then smearing (stout, APE,
HYP), the MatShell product, the FP64 stencil, the plain Krylov-Schur solve, the
covariant displacement, the block solver with every filter variant and the
source shape run with no index out of range, and give the same results as the
normal build.  The checked library runs in a child process (the binding loads
one library per process, chosen by LAPH_GPU_LIB)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _workload(out_path):
    """Everything the checked build is asked to run; the arrays go to out_path (.npz)."""
    import laph_eigsys_b200 as lb
    from conftest import random_links
    res = {}
    rng = np.random.default_rng(5)
    for kind, (p1, p2, it) in {lb.SMEAR_STOUT: (0.1, 0.0, 3), lb.SMEAR_APE: (0.5, 0.0, 4),
                               lb.SMEAR_HYP: (0.62, 0.62, 1)}.items():
        for L in (4, 6):
            c = lb.Context(L, 11.8, 0.6, 8)
            c.set_links(random_links(L, 0.35, 900 + L))
            c.smear(kind, p1, p2, it, 1 if kind != lb.SMEAR_HYP else 0)
            res[f"smear{kind}_{L}"] = c.get_links()
            c.close()
    c = lb.Context(8, 11.8, 0.6, 8)
    U = random_links(8, 0.35, 910)
    c.set_links(U)
    x = rng.normal(size=3 * 8 ** 3) + 1j * rng.normal(size=3 * 8 ** 3)
    res["matmult"] = c.matmult(x)
    res["matmult_d1"] = c.matmult(x, deg=1)
    res["neglap"] = c.apply_neglap(x)
    st, theta, _, nconv, _, _ = c.eps_solve(12, tol=1e-10, max_it=200)
    res["eps_theta"] = theta[:nconv]
    Vr = rng.normal(size=(3 * 8 ** 3, 4)) + 1j * rng.normal(size=(3 * 8 ** 3, 4))
    res["displace"] = c.displace(Vr, 1)
    c.close()
    kw = dict(smear_kind=lb.SMEAR_STOUT, smear_p1=0.1, smear_iters=2, guard=16, tol=1e-10, deg=24)
    for fk, probs in ((0, [(6, 12), (8, 20)]), (1, [(6, 12), (8, 20)]), (2, [(6, 12), (8, 20)]),
                      (3, [(16, 24)]), (4, [(16, 24)]), (5, [(6, 12), (8, 20)])):
        s = lb.Solver(probs, filter_kernel=fk, **kw)
        for i, (L, _) in enumerate(probs):
            s.set_links(i, random_links(L, 0.35, 920 + L))
        st, _ = s.run()
        assert st == 0, (fk, st)
        for i in range(len(probs)):
            ev, Vs, _ = s.get(i)
            res[f"solver{fk}_{i}_ev"] = ev
            if fk == 1 and i == 1:
                res["sourceshape"] = lb.sourceshape(Vs, probs[i][0], ev)
        s.close()
    np.savez(out_path, **res)


def _child(tmp_path):
    """Runs the self-test and the workload in a process with the checked library; returns its report."""
    out = tmp_path / "checked.npz"
    code = (
        "import json, sys\n"
        f"sys.path.insert(0, {HERE!r})\n"
        "import laph_eigsys_b200 as lb\n"
        "import test_gpu_check_build as t\n"
        "assert lb.check_enabled()\n"
        "lb.check_report(reset=True)\n"
        "st = lb.lib.laph_check_selftest(0)\n"
        "selftest = lb.check_report(reset=True)\n"
        f"t._workload({str(out)!r})\n"
        "print(json.dumps({'selftest_status': st, 'selftest': selftest, 'workload': lb.check_report()}))\n")
    env = dict(os.environ, LAPH_GPU_LIB="check")
    p = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stderr[-3000:]
    return json.loads(p.stdout.strip().splitlines()[-1]), np.load(out)


def test_checked_build_finds_no_index_out_of_range_and_matches(tmp_path, gpu):
    rep, checked = _child(tmp_path)
    # the self-test's index 16 + 3 against [0, 16) is recorded, with its bound
    assert rep["selftest_status"] == 0
    assert rep["selftest"]["count"] == 1
    assert rep["selftest"]["index"] == 19 and rep["selftest"]["bound"] == 16
    assert "check.cu" in rep["selftest"]["unit"]
    # nothing else anywhere in the workload
    assert rep["workload"] == {"count": 0}, rep["workload"]
    # the same workload on the normal build
    normal_path = tmp_path / "normal.npz"
    _workload(str(normal_path))
    normal = np.load(normal_path)
    assert sorted(checked.files) == sorted(normal.files)
    for k in checked.files:
        a, b = checked[k], normal[k]
        assert a.shape == b.shape, k
        tol = 1e-10 if (k.startswith("solver") or k.startswith("eps") or k == "sourceshape") else 1e-13
        err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)
        assert err <= tol, (k, err)
