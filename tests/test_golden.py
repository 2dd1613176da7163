"""Committed golden fixtures (tests/golden/make_golden.py): the seeded gauge
generator, the oracle (CPU) and the CUDA path (GPU) reproduce them."""
import os

import numpy as np
import pytest

import laph_eigsys_b200 as lb

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLD, name))


def test_generator_and_oracle_reproduce_fixtures(orc):
    g = load("l4_seed1227.npz")
    L = 4
    conf = lb.gauge_random(L, 2, 0.4, 1227)
    assert np.array_equal(conf, g["conf"])
    U = np.ascontiguousarray(conf[0, :, 1:4])
    assert np.abs(orc.smear_stout(U, L, 0.1, 3, 1) - g["stout_compat"]).max() < 1e-14
    assert np.abs(orc.smear_stout(U, L, 0.1, 3, 0) - g["stout"]).max() < 1e-14
    assert np.abs(orc.smear_ape(U, L, 0.5, 3, 1) - g["ape_compat"]).max() < 1e-14
    Us = orc.smear_hyp(U, L, 0.62, 0.52, 3)
    assert np.abs(Us - g["hyp"]).max() < 1e-14
    assert np.abs(orc.tv_iter(Us, L, 11.8, 0.6, 8, g["x"]) - g["tv_iter_deg8_hyp"]).max() < 1e-11
    assert np.abs(np.linalg.eigvalsh(orc.neglap_dense(Us, L)) - g["neglap_eigs_hyp"]).max() < 1e-12
    f = load("free_spectrum.npz")
    k = 4.0 * np.sin(np.pi * np.arange(6) / 6) ** 2
    assert np.allclose(np.sort(np.repeat((k[:, None, None] + k[None, :, None] + k[None, None, :]).ravel(), 3)),
                       f["L6"], atol=1e-14)


@pytest.mark.gpu
def test_cuda_path_reproduces_fixtures(gpu):
    g = load("l4_seed1227.npz")
    L = 4
    U = np.ascontiguousarray(g["conf"][0, :, 1:4])
    ctx = gpu.Context(L, 11.8, 0.6, 8)
    for name, smear in [("stout_compat", lambda c: c.smearing_stout(0.1, 3, 1)),
                        ("stout", lambda c: c.smearing_stout(0.1, 3, 0)),
                        ("ape_compat", lambda c: c.smearing_ape(0.5, 3, 1)),
                        ("hyp", lambda c: c.smearing_hyp(0.62, 0.52, 3))]:
        ctx.set_links(U)
        smear(ctx)
        got = ctx.get_links()
        rel = np.linalg.norm((got - g[name]).reshape(-1, 9), axis=1) / np.linalg.norm(g[name].reshape(-1, 9), axis=1)
        assert rel.max() <= 1e-12, name
    y = ctx.matmult(g["x"], 8)
    assert np.linalg.norm(y - g["tv_iter_deg8_hyp"]) / np.linalg.norm(g["tv_iter_deg8_hyp"]) <= 1e-13
    assert abs(ctx.plaquette() - float(g["plaquette_hyp"])) < 1e-13
    ctx.close()
    s = gpu.Solver([(L, 20)], guard=16, tol=1e-10, deg=8, max_it=300, smear_kind=gpu.SMEAR_HYP, smear_p1=0.62,
                   smear_p2=0.52,
                   smear_iters=3, link_prec=gpu.LINKS_FP32)
    s.set_links(0, U)
    st, res = s.run()
    assert st == 0
    ev, V, ph = s.get(0)
    assert np.abs(-ev - g["neglap_eigs_hyp"][:20]).max() / 12.0 <= 1e-10
    s.close()


def test_oracle_reproduces_consumer_fixtures(orc):
    """Source shape, radius average and displacement of a stored HYP eigenvector block (l4_hyp_consumers.npz)."""
    g = load("l4_seed1227.npz")
    c = load("l4_hyp_consumers.npz")
    L = 4
    V = c["V"]
    assert np.abs(V.conj().T @ V - np.eye(V.shape[1])).max() < 1e-13
    assert np.abs(orc.sourceshape(V, L) - c["psi"]).max() <= 1e-14 * np.abs(c["psi"]).max()
    r, a = orc.sourceshape_avg(L, c["psi"])
    assert np.array_equal(r, c["radii"]) and np.abs(a - c["psi_avg"]).max() <= 1e-15 * np.abs(a).max()
    for d in range(3):
        assert np.abs(orc.displace(g["hyp"], L, d, V) - c["displaced"][d]).max() < 1e-15
    # psi(0) = sum_x ||V_x V_x^dag||_F, straight from the definition
    p0 = sum(np.linalg.norm(V[3 * x:3 * x + 3] @ V[3 * x:3 * x + 3].conj().T) for x in range(L ** 3))
    assert abs(c["psi"][0] - p0) <= 1e-13 * p0


@pytest.mark.gpu
def test_cuda_consumers_reproduce_fixtures(gpu):
    g = load("l4_seed1227.npz")
    c = load("l4_hyp_consumers.npz")
    L = 4
    V = c["V"]
    psi = gpu.sourceshape(V, L)
    assert np.abs(psi - c["psi"]).max() <= 1e-12 * np.abs(c["psi"]).max()
    ctx = gpu.Context(L, 11.8, 0.6, 8)
    ctx.set_links(g["hyp"])
    for d in range(3):
        W = ctx.displace(V, d)
        assert np.abs(W - c["displaced"][d]).max() <= 1e-14 * np.abs(c["displaced"][d]).max()
    ctx.close()
