"""The bounds-checked build (liblaph_gpu_check.so, the same sources compiled
with -DLAPH_CHECK) loads on a CPU-only host, exports every entry point that
include/laph_gpu.h declares, and says which build it is; the normal build
reports no checked indices and refuses the self-test.  The checked kernels
themselves run in tests/test_gpu_check_build.py."""
import ctypes
import os
import re
import subprocess
import sys

from test_abi import declared_symbols

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECK_SO = os.path.join(ROOT, "laph_eigsys_b200", "liblaph_gpu_check.so")


def test_check_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", CHECK_SO], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(laph_[a-z0-9_]+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing


def test_binding_loads_the_checked_build_on_request():
    code = ("import laph_eigsys_b200 as lb; import os; "
            "print(os.path.basename(lb._lib.LIB_PATH), lb.check_enabled())")
    env = dict(os.environ, LAPH_GPU_LIB="check")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, check=True)
    assert out.stdout.split() == ["liblaph_gpu_check.so", "True"]
    env["LAPH_GPU_LIB"] = "nonsense"
    bad = subprocess.run([sys.executable, "-c", "import laph_eigsys_b200"], cwd=ROOT, env=env, capture_output=True,
                         text=True)
    assert bad.returncode != 0 and "LAPH_GPU_LIB" in bad.stderr


def test_normal_build_reports_nothing_and_refuses_the_self_test():
    import laph_eigsys_b200 as lb
    assert not lb.check_enabled()
    assert lb.check_report() == {"count": 0}
    assert lb.lib.laph_check_selftest(0) == lb._lib.LAPH_EINVAL
    assert b"LAPH_CHECK" in lb.lib.laph_last_error()
    # a NULL count is an argument error in either build
    assert lb.lib.laph_check_report(None, None, None, None, None, 0, 0) == lb._lib.LAPH_EINVAL


def test_checked_build_says_so():
    lib = ctypes.CDLL(CHECK_SO)
    assert lib.laph_check_enabled() == 1
