"""The C-ABI library loads on a CPU-only host and exports every entry point
that include/laph_gpu.h declares (no compute calls)."""
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "laph_gpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(laph_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    import laph_eigsys_b200 as lb
    so = lb._lib.LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", so], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(laph_[a-z0-9_]+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    for s in declared_symbols():
        assert hasattr(lb.lib, s)


def test_version_and_errors():
    import laph_eigsys_b200 as lb
    assert lb.lib.laph_version() >= 100
    assert lb.lib.laph_strerror(0) == b"ok"


def test_sm100a_only():
    """The shipped cubin targets sm_100a."""
    import laph_eigsys_b200 as lb
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", lb._lib.LIB_PATH],
                         capture_output=True, text=True)
    assert "sm_100a" in out.stdout
