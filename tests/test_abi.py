"""The C-ABI library loads on a CPU-only host and exports every entry point
that include/laph_gpu.h declares (no compute calls); on a GPU the runtime
reports its kernels as sm_100 code."""
import os
import re
import subprocess

import pytest

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


@pytest.mark.gpu
def test_kernels_are_built_for_sm100():
    """The CUDA runtime reports the library's kernels as sm_100 code (cudaFuncGetAttributes binaryVersion)."""
    import ctypes
    import laph_eigsys_b200 as lb
    v = ctypes.c_int(0)
    assert lb.lib.laph_binary_version(ctypes.byref(v)) == 0, lb.lib.laph_last_error()
    assert v.value == 100


def test_binary_version_without_a_device_is_an_error_not_a_guess():
    import ctypes
    import torch
    import laph_eigsys_b200 as lb
    if torch.cuda.is_available():
        pytest.skip("a device is visible")
    v = ctypes.c_int(-1)
    assert lb.lib.laph_binary_version(ctypes.byref(v)) != 0
    assert v.value == -1


@pytest.mark.gpu
def test_fp64_probe_measures_plausible_peaks():
    """laph_probe_fp64 (the FP64 rooflines' denominators, measured in place) gives B200-sized figures: tens of
    TFLOP/s on the FMA pipe and on the FP64 tensor path."""
    import laph_eigsys_b200 as lb
    fma, dmma = lb.probe_fp64(0)
    assert 10.0 < fma < 120.0 and 10.0 < dmma < 120.0, (fma, dmma)


def test_solve_opts_mirror_matches_the_c_struct():
    """laph_solve_opts_default writes the C struct: it must end exactly where the ctypes mirror ends (a sentinel
    just past it stays untouched) and its last field, direct_resid, must read back as the library's default."""
    import ctypes
    import laph_eigsys_b200 as lb
    n = ctypes.sizeof(lb._lib.laph_solve_opts)
    buf = (ctypes.c_ubyte * (n + 64))(*([0xA5] * (n + 64)))
    lb.lib.laph_solve_opts_default(ctypes.cast(buf, ctypes.POINTER(lb._lib.laph_solve_opts)))
    assert bytes(buf[n:]) == b"\xa5" * 64
    o = lb._lib.laph_solve_opts.from_buffer(buf)
    assert o.direct_resid == 1e-3 and o.filter_kernel == 1 and o.guard == 16 and o.max_it == 200
