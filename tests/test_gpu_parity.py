"""CUDA path vs the FP64 oracle: smearing (<= 1e-12 relative per link) and the
MatShell MatMult body T_deg(B) x (<= 1e-13 relative), through the C ABI."""
import numpy as np
import pytest

from conftest import random_links, unit_links

pytestmark = pytest.mark.gpu


def rel_link_err(A, B):
    a = A.reshape(-1, 9)
    b = B.reshape(-1, 9)
    return (np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)).max()


@pytest.mark.parametrize("L", [4, 6, 8])
@pytest.mark.parametrize("kind,p1,p2,it,compat", [
    ("stout", 0.1, 0.0, 3, 1), ("stout", 0.1, 0.0, 5, 0), ("ape", 0.5, 0.0, 3, 1), ("ape", 0.5, 0.0, 2, 0),
    ("hyp", 0.62, 0.52, 3, 0), ("hyp", 0.62, 0.62, 1, 0)])
def test_smearing_parity(gpu, orc, L, kind, p1, p2, it, compat):
    U = random_links(L, 0.4, 1227 + L)
    ctx = gpu.Context(L)
    ctx.set_links(U)
    if kind == "stout":
        ctx.smearing_stout(p1, it, compat)
        ref = orc.smear_stout(U, L, p1, it, compat)
    elif kind == "ape":
        ctx.smearing_ape(p1, it, compat)
        ref = orc.smear_ape(U, L, p1, it, compat)
    else:
        ctx.smearing_hyp(p1, p2, it)
        ref = orc.smear_hyp(U, L, p1, p2, it)
    got = ctx.get_links()
    assert rel_link_err(got, ref) <= 1e-12
    ctx.close()


def test_link_layouts_roundtrip(gpu):
    L = 4
    U = random_links(L, 0.4, 9)
    ctx = gpu.Context(L)
    ctx.set_links(U, gpu.LAYOUT_ROWMAJOR)
    E = ctx.get_links(gpu.LAYOUT_EIGEN)
    assert np.array_equal(E, np.transpose(U, (0, 1, 3, 2)))
    ctx.set_links(E, gpu.LAYOUT_EIGEN)
    assert np.array_equal(ctx.get_links(), U)
    conf = gpu.gauge_random(L, 1, 0.4, 3)[0]
    ctx.set_links(conf, gpu.LAYOUT_CONF)
    assert np.array_equal(ctx.get_links(), conf[:, 1:4])


@pytest.mark.parametrize("L", [4, 8, 12])
@pytest.mark.parametrize("deg", [1, 2, 3, 8, 12])
def test_matmult_parity(gpu, orc, L, deg):
    U = orc.smear_hyp(random_links(L, 0.4, 1300 + L), L, 0.62, 0.52, 1)
    lam_l, lam_c = 11.8, 0.6
    ctx = gpu.Context(L, lam_l, lam_c, deg)
    ctx.set_links(U)
    rng = np.random.default_rng(L * 100 + deg)
    x = rng.normal(size=3 * L ** 3) + 1j * rng.normal(size=3 * L ** 3)
    y = ctx.matmult(x)
    ref = orc.tv2(U, L, lam_l, lam_c, x) if deg == 1 else orc.tv_iter(U, L, lam_l, lam_c, deg, x)
    assert np.linalg.norm(y - ref) / np.linalg.norm(ref) <= 1e-13
    ctx.close()


@pytest.mark.parametrize("L,deg", [(32, 12), (16, 9), (24, 8), (36, 5), (5, 7)])
def test_matmult_fused_launch_shapes(gpu, orc, L, deg):
    """The one-launch product at the largest lattice whose sites all fit the device's co-resident CTAs one per
    thread (32^3: 256 CTAs, links held in registers and shared memory), at 16^3 and 24^3, beyond co-residency
    (36^3: grid-stride, links read per step) and at a ragged last CTA (5^3 = 125 sites), against the oracle's
    tv_iter, through host and device pointers, twice in a row on one context."""
    import torch
    U = random_links(L, 0.3, 1500 + L)
    lam_l, lam_c = 12.0, 0.7
    ctx = gpu.Context(L, lam_l, lam_c, deg)
    ctx.set_links(U)
    rng = np.random.default_rng(L)
    for rep in range(2):
        x = rng.normal(size=3 * L ** 3) + 1j * rng.normal(size=3 * L ** 3)
        ref = orc.tv_iter(U, L, lam_l, lam_c, deg, x)
        y = ctx.matmult(x)
        assert np.linalg.norm(y - ref) / np.linalg.norm(ref) <= 1e-13, (rep, "host")
        dx = torch.from_numpy(x.copy()).cuda()
        dy = torch.empty_like(dx)
        ctx.matmult_device(dx.data_ptr(), dy.data_ptr())
        yd = dy.cpu().numpy()
        assert np.linalg.norm(yd - ref) / np.linalg.norm(ref) <= 1e-13, (rep, "device")
    # overlapping device vectors are refused: the product reads x while it writes y
    with pytest.raises(gpu.LaphError) as e:
        ctx.matmult_device(dx.data_ptr(), dx.data_ptr())
    assert e.value.status == gpu._lib.LAPH_EINVAL
    ctx.close()


def test_neglap_diag_plaquette(gpu, orc):
    L = 6
    U = random_links(L, 0.4, 77)
    ctx = gpu.Context(L)
    ctx.set_links(U)
    rng = np.random.default_rng(1)
    x = rng.normal(size=3 * L ** 3) + 1j * rng.normal(size=3 * L ** 3)
    y = ctx.apply_neglap(x)
    ref = orc.neglap(U, L, x)
    assert np.linalg.norm(y - ref) / np.linalg.norm(ref) <= 1e-14
    assert np.all(ctx.get_diagonal() == -6.0)
    assert abs(ctx.plaquette() - orc.plaquette(U, L)) < 1e-13
    ctx.set_links(unit_links(L))
    assert abs(ctx.plaquette() - 1.0) < 1e-15


def test_matmult_rejects_bad_window(gpu):
    ctx = gpu.Context(4, 1.0, 2.0, 8)
    with pytest.raises(gpu.LaphError):
        ctx.matmult(np.zeros(3 * 64, dtype=np.complex128))


def test_non_finite_links_are_refused_on_the_host(gpu, orc):
    """NaN or Inf in a spatial link is refused by laph_set_links / laph_solver_set_links before any device work
    (LAPH_EINVAL naming the site); the context and the solver stay usable with good links."""
    L = 4
    U = random_links(L, 0.4, 78)
    for bad_value, site in ((np.nan, 5), (np.inf, 0), (-np.inf, L ** 3 - 1)):
        Ub = U.copy()
        Ub[site, 1, 2, 0] = bad_value
        ctx = gpu.Context(L)
        with pytest.raises(gpu.LaphError) as e:
            ctx.set_links(Ub)
        assert e.value.status == gpu._lib.LAPH_EINVAL and f"site {site}" in str(e.value)
        ctx.set_links(U)
        assert abs(ctx.plaquette() - orc.plaquette(U, L)) < 1e-13
        ctx.close()
        s = gpu.Solver([(L, 8)], tol=1e-10, deg=8)
        with pytest.raises(gpu.LaphError) as e:
            s.set_links(0, Ub)
        assert e.value.status == gpu._lib.LAPH_EINVAL
        s.set_links(0, U)
        st, _ = s.run()
        assert st == 0
        s.close()

