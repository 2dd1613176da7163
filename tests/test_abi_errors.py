"""C-ABI argument checking on a CPU-only host: every entry point rejects bad
arguments with LAPH_EINVAL and a message naming it, before touching a device;
well-formed calls without a CUDA device return LAPH_ENODEV (never a host
fallback); null handles are rejected and destroying a null handle is a no-op."""
import ctypes

import numpy as np
import pytest

from laph_eigsys_b200 import _lib
from laph_eigsys_b200._lib import laph_params, laph_problem, laph_solve_opts, lib


def _has_device():
    import torch
    return torch.cuda.is_available()


def _err():
    return lib.laph_last_error().decode()


def _opts(**kw):
    o = laph_solve_opts()
    lib.laph_solve_opts_default(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def _solver_create(probs, n=None, **kw):
    arr = (laph_problem * max(len(probs), 1))(*[laph_problem(L, nev) for L, nev in probs])
    h = ctypes.c_void_p()
    o = _opts(**kw)
    st = lib.laph_solver_create(ctypes.byref(h), arr, len(probs) if n is None else n, ctypes.byref(o), 0)
    if st == _lib.LAPH_OK:
        lib.laph_solver_destroy(h)
    return st


@pytest.mark.parametrize("probs,kw", [
    ([(8, 10)], {"deg": 1}),
    ([(8, 10)], {"deg": 129}),
    ([(8, 10)], {"guard": -1}),
    ([(8, 10)], {"tol": 0.0}),
    ([(8, 10)], {"tol": float("nan")}),
    ([(8, 10)], {"max_it": 0}),
    ([(8, 10)], {"block": 513}),
    ([(8, 10)], {"filter_kernel": 6}),
    ([(8, 10)], {"filter_kernel": -1}),
    ([(8, 10)], {"direct_resid": float("nan")}),
    ([(8, 10)], {"direct_resid": float("inf")}),
    ([(2, 1)], {}),
    ([(129, 10)], {}),
    ([(8, 0)], {}),
    ([(3, 40)], {}),              # block width 64 > dim / 2 = 40
    ([(32, 500)], {}),            # block width 544 > 512
    ([(8, 10), (4, 90)], {}),     # the second problem: block width 128 > dim / 2 = 96
])
def test_solver_create_rejects_bad_arguments(probs, kw):
    assert _solver_create(probs, **kw) == _lib.LAPH_EINVAL
    assert _err().startswith("laph_solver_create")


def test_solver_create_null_and_empty():
    o = _opts()
    h = ctypes.c_void_p()
    arr = (laph_problem * 1)(laph_problem(8, 10))
    assert lib.laph_solver_create(None, arr, 1, ctypes.byref(o), 0) == _lib.LAPH_EINVAL
    assert lib.laph_solver_create(ctypes.byref(h), None, 1, ctypes.byref(o), 0) == _lib.LAPH_EINVAL
    assert lib.laph_solver_create(ctypes.byref(h), arr, 0, ctypes.byref(o), 0) == _lib.LAPH_EINVAL
    assert lib.laph_solver_create(ctypes.byref(h), arr, 1, None, 0) == _lib.LAPH_EINVAL


def test_well_formed_calls_without_device_report_enodev():
    if _has_device():
        pytest.skip("a device is present")
    assert _solver_create([(8, 10), (6, 12)]) == _lib.LAPH_ENODEV
    assert "no CUDA device" in _err()
    h = ctypes.c_void_p()
    p = laph_params(8, 12.0, 0.6, 8, 0)
    assert lib.laph_ctx_create(ctypes.byref(h), ctypes.byref(p)) == _lib.LAPH_ENODEV
    L, nev = 4, 3
    V = np.zeros((3 * L ** 3, nev), dtype=np.complex128, order="F")
    psi = np.empty((L // 2) ** 3)
    st = lib.laph_sourceshape(ctypes.c_void_p(V.ctypes.data), L, nev, None, 0, ctypes.c_void_p(psi.ctypes.data), 0)
    assert st == _lib.LAPH_ENODEV


def test_ctx_create_rejects_bad_arguments():
    h = ctypes.c_void_p()
    for L in (2, 513):
        p = laph_params(L, 12.0, 0.6, 8, 0)
        assert lib.laph_ctx_create(ctypes.byref(h), ctypes.byref(p)) == _lib.LAPH_EINVAL
    assert lib.laph_ctx_create(ctypes.byref(h), None) == _lib.LAPH_EINVAL
    assert lib.laph_ctx_create(None, ctypes.byref(laph_params(8, 12.0, 0.6, 8, 0))) == _lib.LAPH_EINVAL


def test_null_handles():
    assert lib.laph_ctx_destroy(None) == _lib.LAPH_OK
    assert lib.laph_solver_destroy(None) == _lib.LAPH_OK
    assert lib.laph_solver_run(None, None) == _lib.LAPH_EINVAL
    buf = np.zeros(16)
    p = ctypes.c_void_p(buf.ctypes.data)
    assert lib.laph_displace(None, 0, p, p, 1, 0) == _lib.LAPH_EINVAL
    assert lib.laph_solver_displace(None, 0, 0, p, 0) == _lib.LAPH_EINVAL
    assert lib.laph_solver_sourceshape(None, 0, 0, p) == _lib.LAPH_EINVAL


def test_displace_rejects_bad_direction_and_sizes():
    buf = np.zeros(16)
    p = ctypes.c_void_p(buf.ctypes.data)
    for d, nev in ((-1, 1), (3, 1), (0, 0)):
        assert lib.laph_displace(None, d, p, p, nev, 0) == _lib.LAPH_EINVAL
        assert _err().startswith("laph_displace")
    assert lib.laph_displace(None, 0, None, p, 1, 0) == _lib.LAPH_EINVAL


def test_matmult_noalloc_rejects_bad_arguments():
    buf = np.zeros(2 * 3 * 8 ** 3)
    p = ctypes.c_void_p(buf.ctypes.data)
    f = lib.laph_matmult_noalloc
    assert f(None, 8, 12.0, 0.6, 8, p, p, None) == _lib.LAPH_EINVAL
    assert f(p, 8, 12.0, 0.6, 8, None, p, None) == _lib.LAPH_EINVAL
    for L in (2, 33):
        assert f(p, L, 12.0, 0.6, 8, p, p, None) == _lib.LAPH_EINVAL
    assert "scratch" in _err()
    assert f(p, 8, 12.0, 0.6, 0, p, p, None) == _lib.LAPH_EINVAL
    assert f(p, 8, 0.6, 12.0, 8, p, p, None) == _lib.LAPH_EINVAL


def test_sourceshape_rejects_bad_arguments():
    V = np.zeros((3 * 64, 2), dtype=np.complex128)
    psi = np.empty(8)
    pv, pp = ctypes.c_void_p(V.ctypes.data), ctypes.c_void_p(psi.ctypes.data)
    for args in ((None, 4, 2), (pv, 5, 2), (pv, 0, 2), (pv, 4, 0)):
        assert lib.laph_sourceshape(args[0], args[1], args[2], None, 0, pp, 0) == _lib.LAPH_EINVAL
        assert _err().startswith("laph_sourceshape")
    assert lib.laph_sourceshape(pv, 4, 2, None, 0, None, 0) == _lib.LAPH_EINVAL
    r, a = np.empty(8), np.empty(8)
    n = ctypes.c_int()
    for L in (0, 3):
        assert lib.laph_sourceshape_avg(L, pp, ctypes.c_void_p(r.ctypes.data), ctypes.c_void_p(a.ctypes.data),
                                        ctypes.byref(n)) == _lib.LAPH_EINVAL


def test_timeslice_split_rejects_bad_arguments():
    t0, c = ctypes.c_int(), ctypes.c_int()
    for LT, size, rank in ((-1, 1, 0), (4, 0, 0), (4, 2, 2), (4, 2, -1)):
        assert lib.laph_timeslice_split(LT, size, rank, ctypes.byref(t0), ctypes.byref(c)) == _lib.LAPH_EINVAL
    assert lib.laph_timeslice_split(0, 3, 2, ctypes.byref(t0), ctypes.byref(c)) == _lib.LAPH_OK
    assert c.value == 0


def test_mlp_forward_rejects_bad_arguments():
    x = np.zeros(64, dtype=np.float32)
    p = ctypes.c_void_p(x.ctypes.data)
    assert lib.laph_mlp_forward(None, p, 1, p, 0) == _lib.LAPH_EINVAL
    assert lib.laph_mlp_forward(p, p, 0, p, 0) == _lib.LAPH_EINVAL


def test_last_error_is_per_thread():
    """Each thread reads back the message of its own failing call, however the calls interleave."""
    import threading
    import time
    errors = {}

    def worker(k):
        for it in range(200):
            if k % 2:
                st = lib.laph_timeslice_split(-k, 1, 0, None, None)
                want = "laph_timeslice_split"
            else:
                st = lib.laph_reset_phase_host(0, 1, None, None, None)
                want = "laph_reset_phase_host"
            time.sleep(0)
            msg = lib.laph_last_error().decode()
            if st != _lib.LAPH_EINVAL or not msg.startswith(want):
                errors[k] = (it, st, msg)
                return

    ts = [threading.Thread(target=worker, args=(k,)) for k in range(8)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errors, errors


def test_noalloc_refuses_overlapping_vectors_before_the_device():
    """laph_matmult_noalloc reads x while it writes y, so overlapping x and y are refused with LAPH_EINVAL before
    any CUDA call (the pointers below are never dereferenced)."""
    L = 4
    vb = 16 * 3 * L ** 3
    base = 1 << 40
    for dx, dy in ((base, base), (base, base + vb - 16), (base + 32, base)):
        st = lib.laph_matmult_noalloc(ctypes.c_void_p(base), L, 12.0, 0.5, 4, ctypes.c_void_p(dx),
                                      ctypes.c_void_p(dy), None)
        assert st == _lib.LAPH_EINVAL, (dx, dy)
        assert "overlap" in _err()
    # L beyond the fixed array, deg < 1 and a reversed window are refused the same way
    for L_, deg, ll, lc in ((33, 4, 12.0, 0.5), (8, 0, 12.0, 0.5), (8, 4, 0.5, 12.0)):
        st = lib.laph_matmult_noalloc(ctypes.c_void_p(base), L_, ll, lc, deg, ctypes.c_void_p(base),
                                      ctypes.c_void_p(base + (1 << 30)), None)
        assert st == _lib.LAPH_EINVAL
