"""The autotuner's search on CPU with synthetic trial costs (axis order, the 1%
margin, failed settings, no setting timed twice), its argument checks, and that
without a device it stops with LAPH_ENODEV."""
import ctypes

import numpy as np
import pytest

import laph_eigsys_b200 as lb
from laph_eigsys_b200 import _lib

DEGS, BLOCKS, GUARDS = [40, 48, 56, 60, 64], [16, 32, 64], [16, 48]


def _cost(d, b, g):
    return 100.0 + 0.5 * (d - 56) ** 2 + 3.0 * abs(np.log2(b / 32)) + (4.0 if g == 48 else 0.0)


def test_search_finds_separable_optimum_and_times_each_setting_once():
    seen = []

    def trial(d, b, g):
        seen.append((d, b, g))
        return _cost(d, b, g)

    r = lb.autotune_search(DEGS, BLOCKS, GUARDS, (60, 32, 16), trial)
    assert (r["deg"], r["block"], r["guard"]) == (56, 32, 16)
    assert r["ms_per_problem"] == _cost(56, 32, 16) and r["from_cache"] == 0
    assert len(seen) == len(set(seen)) == r["trials"] == 1 + 4 + 2 + 1
    # axis order: every deg candidate before any block candidate, blocks before guards
    assert [s for s in seen if s[1] != 32 or s[2] != 16] == [(56, 16, 16), (56, 64, 16), (56, 32, 48)]


def test_search_margin_keeps_start_against_noise():
    # 0.5% faster is noise; 2% faster is taken
    r = lb.autotune_search([48], [], [], (60, 32, 16), lambda d, b, g: 100.0 if d == 60 else 99.5)
    assert r["deg"] == 60 and r["ms_per_problem"] == 100.0
    r = lb.autotune_search([48], [], [], (60, 32, 16), lambda d, b, g: 100.0 if d == 60 else 98.0)
    assert r["deg"] == 48


def test_search_skips_failed_settings():
    # the start fails (e.g. no convergence within max_it); the first working candidate wins outright
    r = lb.autotune_search(DEGS, BLOCKS, [], (16, 32, 16),
                           lambda d, b, g: -1.0 if d < 48 or b == 64 else _cost(d, b, g))
    assert (r["deg"], r["block"]) == (56, 32)
    with pytest.raises(lb.LaphError) as e:
        lb.autotune_search(DEGS, BLOCKS, GUARDS, (60, 32, 16), lambda d, b, g: float("nan"))
    assert e.value.status == _lib.LAPH_ENOTCONV


def test_argument_checks_and_no_device():
    r = _lib.laph_tune_result()
    assert lib_call(lambda: lb.lib.laph_autotune_search(None, 2, None, 0, None, 0, 60, 32, 16,
                                                        _lib.TUNE_TRIAL(lambda *a: 1.0), None, ctypes.byref(r))) == \
        _lib.LAPH_EINVAL
    with pytest.raises(lb.LaphError) as e:
        lb.autotune([(8, 20)], [], nsample=0)
    assert e.value.status == _lib.LAPH_EINVAL
    U0 = np.zeros((8 ** 3, 3, 3, 3), dtype=np.complex128)
    with pytest.raises(lb.LaphError) as e:  # the learned window needs its model for the trial solves
        lb.autotune([(8, 20)], [U0], window=lb.WINDOW_MLP)
    assert e.value.status == _lib.LAPH_EINVAL and "model" in str(e.value)
    import torch
    if not torch.cuda.is_available():
        U = np.zeros((8 ** 3, 3, 3, 3), dtype=np.complex128)
        with pytest.raises(lb.LaphError) as e:
            lb.autotune([(8, 20)], [U])
        assert e.value.status == _lib.LAPH_ENODEV


def lib_call(f):
    return f()


def test_solver_footprint_arithmetic():
    """The footprint the wave planner uses: additive over equal problems up to the shared buffers, monotone, and
    the 48^3 x 96, nev 220 batch (about 7 GB per timeslice) does not fit one 180 GB device."""
    kw = dict(guard=16, deg=48)
    one = lb.solver_footprint([(48, 220)], **kw)
    assert 6.5e9 < one < 8e9
    assert lb.solver_footprint([(48, 220)] * 96, **kw) > 180e9
    sizes = [lb.solver_footprint([(32, 120)] * m, guard=16, deg=60) for m in (1, 2, 4, 8, 64)]
    assert all(a < b for a, b in zip(sizes, sizes[1:]))
    per = (sizes[3] - sizes[2]) / 4
    assert abs((sizes[4] - sizes[3]) / 56 - per) <= 1e-3 * per  # linear in the number of equal problems
    assert lb.solver_footprint([(8, 20), (16, 60)]) > lb.solver_footprint([(16, 60)])
    for bad in ([(2, 1)], [(129, 10)], [(4, 90)]):
        with pytest.raises(lb.LaphError) as e:
            lb.solver_footprint(bad)
        assert e.value.status == _lib.LAPH_EINVAL
    import torch
    if not torch.cuda.is_available():
        with pytest.raises(lb.LaphError) as e:
            lb.solver_max_batch([(32, 120)] * 4)
        assert e.value.status == _lib.LAPH_ENODEV
    with pytest.raises(lb.LaphError) as e:
        lb.solver_max_batch([(32, 120)], fraction=0.0)
    assert e.value.status == _lib.LAPH_EINVAL
