"""laph_matmult_noalloc: the FP64 MatShell product for callers that cannot
allocate device memory (inside another library's stream capture, under a
framework that owns the device memory budget).  Its Chebyshev temporaries
live in a fixed device array inside the library, so the test checks it
through the C ABI against the allocating entry point laph_matmult, on two
calls in a row (the array keeps the previous call's contents), and that a
timeslice larger than the array is refused.  This file sorts last so that a
run stopping at the first failure has run every other test first."""
import ctypes

import numpy as np
import pytest

from conftest import random_links

pytestmark = pytest.mark.gpu


def _call(lib, dU, L, lam_l, lam_c, deg, dx, dy, stream):
    return lib.laph_matmult_noalloc(ctypes.c_void_p(dU.data_ptr()), L, lam_l, lam_c, deg,
                                    ctypes.c_void_p(dx.data_ptr()), ctypes.c_void_p(dy.data_ptr()),
                                    ctypes.c_void_p(stream))


def test_noalloc_matches_matmult_on_two_calls(gpu):
    import torch
    lib = gpu.lib
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(11)
    for call, (L, deg, lam_l, lam_c) in enumerate([(8, 8, 11.8, 0.6), (12, 5, 12.0, 0.9)]):
        U = random_links(L, 0.4, 4000 + call)
        ctx = gpu.Context(L, lam_l, lam_c, deg)
        ctx.set_links(U)
        x = rng.normal(size=3 * L ** 3) + 1j * rng.normal(size=3 * L ** 3)
        y_ref = ctx.matmult(x)
        ctx.close()
        dU = torch.from_numpy(np.ascontiguousarray(U).view(np.float64).copy()).cuda()
        dx = torch.from_numpy(x.view(np.float64).copy()).cuda()
        dy = torch.full_like(dx, float("nan"))
        assert _call(lib, dU, L, lam_l, lam_c, deg, dx, dy, stream) == 0, lib.laph_last_error()
        torch.cuda.synchronize()
        y = dy.cpu().numpy().view(np.complex128)
        rel = np.linalg.norm(y - y_ref) / np.linalg.norm(y_ref)
        assert rel <= 1e-13, (call, rel)


def test_noalloc_rejects_sizes_beyond_its_array(gpu):
    import torch
    lib = gpu.lib
    d = torch.zeros(8, dtype=torch.float64, device="cuda")
    st = _call(lib, d, 33, 12.0, 0.5, 4, d, d, 0)
    assert st == gpu._lib.LAPH_EINVAL
    assert b"32" in lib.laph_last_error()
