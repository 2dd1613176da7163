import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs through liblaph_gpu.so")


def random_links(L, eps=0.4, seed=1227, ts=0):
    """Spatial links (V3, 3, 3, 3) of timeslice ts of the seeded synthetic field."""
    import laph_eigsys_b200 as lb
    conf = lb.gauge_random(L, ts + 1, eps, seed)
    return np.ascontiguousarray(conf[ts, :, 1:4])


def unit_links(L):
    U = np.zeros((L ** 3, 3, 3, 3), dtype=np.complex128)
    U[:, :, 0, 0] = U[:, :, 1, 1] = U[:, :, 2, 2] = 1.0
    return U


def random_su3_field(L, seed):
    """Random SU(3) gauge transformation Omega(x) (V3, 3, 3) from the seeded generator."""
    import laph_eigsys_b200 as lb
    conf = lb.gauge_random(L, 1, 2.0, seed)
    return np.ascontiguousarray(conf[0, :, 0])


def pure_gauge_links(L, Omega):
    """U_mu(x) = Omega(x)^dag Omega(x+mu) (config_utils.cpp:447-472)."""
    V3 = L ** 3
    U = np.empty((V3, 3, 3, 3), dtype=np.complex128)
    s = np.arange(V3)
    x, y, z = s // (L * L), (s // L) % L, s % L
    ups = [((x + 1) % L) * L * L + y * L + z, x * L * L + ((y + 1) % L) * L + z, x * L * L + y * L + (z + 1) % L]
    for mu in range(3):
        U[:, mu] = np.conj(np.transpose(Omega, (0, 2, 1))) @ Omega[ups[mu]]
    return U


@pytest.fixture(scope="session")
def orc():
    import oracle
    return oracle


@pytest.fixture(scope="session")
def gpu():
    """Skip unless a CUDA device is visible; the product path itself has no fallback."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import laph_eigsys_b200 as lb
    return lb
