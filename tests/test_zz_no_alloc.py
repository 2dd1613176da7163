"""laph_matmult_noalloc: the FP64 MatShell product for callers that may not
allocate device memory where they need it (a framework that owns the device
memory budget through its own pool, a service that allocates only at
start-up).  Its Chebyshev temporaries live in a fixed device array inside the
library, shared by every call and keeping the previous call's contents, so
the test makes consecutive calls through the C ABI and checks each one
against the CPU oracle's tv_iter / tv2 (modules/shell_matop.cpp:16-168) and
against the allocating entry point laph_matmult, at the MatMult tolerance of
the other parity tests (1e-13 relative).  It also checks that a repeated call
leaves the device's free memory where it was, and that a timeslice larger
than the array is refused.  This file sorts last so that a run stopping at
the first failure has run every other test first."""
import ctypes

import numpy as np
import pytest

from conftest import random_links

pytestmark = pytest.mark.gpu

# (L, deg, LAM_L, LAM_C): deg 1 is tv2 alone; 5 and 8 leave T_deg in the array's other slots
CASES = [(8, 8, 11.8, 0.6), (12, 5, 12.0, 0.9), (6, 1, 11.8, 0.6), (8, 7, 11.8, 0.6)]


def _call(lib, dU, L, lam_l, lam_c, deg, dx, dy, stream):
    return lib.laph_matmult_noalloc(ctypes.c_void_p(dU.data_ptr()), L, lam_l, lam_c, deg,
                                    ctypes.c_void_p(dx.data_ptr()), ctypes.c_void_p(dy.data_ptr()),
                                    ctypes.c_void_p(stream))


def test_noalloc_matches_oracle_and_matmult_on_consecutive_calls(gpu, orc):
    import torch
    lib = gpu.lib
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(11)
    for call, (L, deg, lam_l, lam_c) in enumerate(CASES):
        U = random_links(L, 0.4, 4000 + call)
        x = rng.normal(size=3 * L ** 3) + 1j * rng.normal(size=3 * L ** 3)
        y_orc = orc.tv2(U, L, lam_l, lam_c, x) if deg == 1 else orc.tv_iter(U, L, lam_l, lam_c, deg, x)
        ctx = gpu.Context(L, lam_l, lam_c, deg)
        ctx.set_links(U)
        y_mm = ctx.matmult(x)
        ctx.close()
        dU = torch.from_numpy(np.ascontiguousarray(U).view(np.float64).copy()).cuda()
        dx = torch.from_numpy(x.view(np.float64).copy()).cuda()
        dy = torch.full_like(dx, float("nan"))
        assert _call(lib, dU, L, lam_l, lam_c, deg, dx, dy, stream) == 0, lib.laph_last_error()
        torch.cuda.synchronize()
        y = dy.cpu().numpy().view(np.complex128)
        rel_orc = np.linalg.norm(y - y_orc) / np.linalg.norm(y_orc)
        rel_mm = np.linalg.norm(y - y_mm) / np.linalg.norm(y_mm)
        assert rel_orc <= 1e-13, (call, L, deg, rel_orc)
        assert rel_mm <= 1e-13, (call, L, deg, rel_mm)
        # the same call again: no device memory taken or given back, same result
        free0 = torch.cuda.mem_get_info()[0]
        dy.fill_(float("nan"))
        assert _call(lib, dU, L, lam_l, lam_c, deg, dx, dy, stream) == 0, lib.laph_last_error()
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0, call
        assert np.array_equal(dy.cpu().numpy().view(np.complex128), y), call


def test_noalloc_rejects_sizes_beyond_its_array(gpu):
    import torch
    lib = gpu.lib
    d = torch.zeros(8, dtype=torch.float64, device="cuda")
    e = torch.zeros(8, dtype=torch.float64, device="cuda")
    st = _call(lib, d, 33, 12.0, 0.5, 4, d, e, 0)
    assert st == gpu._lib.LAPH_EINVAL
    assert b"32" in lib.laph_last_error()
