"""Source shape psi(r) (the reference's sourceshape program): the device kernel
against the oracle's restatement of source_shape_complete, the radius average
and the output files; analytic checks on the free field."""
import os
import subprocess
import sys

import numpy as np
import pytest

import laph_eigsys_b200 as lb
from conftest import random_links, unit_links


def test_avg_and_writers_match_oracle(orc, tmp_path):
    L = 8
    rng = np.random.default_rng(3)
    psi = rng.uniform(1.0, 2.0, size=(L // 2) ** 3)
    r, a = lb.sourceshape_avg(L, psi)
    ro, ao = orc.sourceshape_avg(L, psi)
    assert np.array_equal(r, ro) and np.allclose(a, ao, rtol=0, atol=1e-15)
    # radii appear in the order of the r1-outer, r3-inner loop and are all distinct
    assert r[0] == 0.0 and r[1] == 2.0 and len(set(np.round(r, 9))) == len(r)
    lb.write_sourceshape(tmp_path, 1227, 5, 40, r, a)
    txt = open(tmp_path / "sourceshape_nev40.1227.5").read().splitlines()
    assert txt[0] == "#r\tpsi(r)" and len(txt) == len(r) + 1
    assert all(abs(float(ln.split()[1]) - v) <= 1e-11 * abs(v) for ln, v in zip(txt[1:], a))
    raw = np.fromfile(tmp_path / "sourceshape_nev40.1227.005.bin", dtype=np.float64).reshape(-1, 2)
    assert np.array_equal(raw[:, 0], r) and np.array_equal(raw[:, 1], a)


def test_oracle_free_field_shape(orc):
    """Unit links: the nev = 3 lowest eigenvectors are the constant modes, V_x = I / sqrt(V3) up to a unitary mix,
    so every 3x3 block is I / V3 and psi(r) = V3 * sqrt(3) / V3 = sqrt(3) for every r."""
    L = 4
    V3 = L ** 3
    V = np.zeros((3 * V3, 3), dtype=np.complex128)
    for c in range(3):
        V[c::3, c] = 1.0 / np.sqrt(V3)
    Q, _ = np.linalg.qr(np.random.default_rng(0).normal(size=(3, 3)) + 1j)
    psi = orc.sourceshape(V @ Q, L)
    assert np.allclose(psi, np.sqrt(3.0), rtol=0, atol=1e-13)


@pytest.mark.gpu
@pytest.mark.parametrize("L,nev", [(4, 6), (6, 20), (8, 40)])
def test_sourceshape_kernel_matches_oracle(gpu, orc, L, nev):
    rng = np.random.default_rng(L)
    V = rng.normal(size=(3 * L ** 3, nev)) + 1j * rng.normal(size=(3 * L ** 3, nev))
    V, _ = np.linalg.qr(V)
    ev = -np.sort(rng.uniform(0.1, 2.0, nev))
    psi = gpu.sourceshape(V, L)
    ref = orc.sourceshape(V, L)
    assert np.abs(psi - ref).max() <= 1e-12 * np.abs(ref).max()
    psiw = gpu.sourceshape(V, L, evals=ev)
    refw = orc.sourceshape(V * np.sqrt(np.abs(ev))[None, :], L)
    assert np.abs(psiw - refw).max() <= 1e-12 * np.abs(refw).max()


@pytest.mark.gpu
def test_solver_sourceshape_on_device(gpu, orc):
    """The solver's own block, in place on the device, against the oracle on the fetched eigenvectors."""
    L, nev = 8, 30
    U = random_links(L, 0.4, 77)
    s = gpu.Solver([(L, nev), (6, 12)], tol=1e-10, deg=8, max_it=300, link_prec=gpu.LINKS_FP32)
    s.set_links(0, U)
    s.set_links(1, random_links(6, 0.4, 78))
    st, _ = s.run()
    assert st == 0
    ev, V, _ = s.get(0)
    psi = s.sourceshape(0)
    ref = orc.sourceshape(V, L)
    assert np.abs(psi - ref).max() <= 1e-12 * np.abs(ref).max()
    psiw = s.sourceshape(0, weighted=True)
    refw = orc.sourceshape(V * np.sqrt(np.abs(ev))[None, :], L)
    assert np.abs(psiw - refw).max() <= 1e-12 * np.abs(refw).max()
    # psi(0) = sum_x ||V_x V_x^dag||_F is the same for every unitary mix of the block
    psi1 = s.sourceshape(1)
    ev1, V1, _ = s.get(1)
    assert np.abs(psi1 - orc.sourceshape(V1, 6)).max() <= 1e-12 * np.abs(psi1).max()
    s.close()


@pytest.mark.gpu
def test_sourceshape_free_field_gpu(gpu):
    """Unit gauge field: psi(r) = sqrt(3) for the 3 constant modes."""
    L = 8
    V3 = L ** 3
    V = np.zeros((3 * V3, 3), dtype=np.complex128)
    for c in range(3):
        V[c::3, c] = 1.0 / np.sqrt(V3)
    assert np.allclose(gpu.sourceshape(V, L), np.sqrt(3.0), rtol=0, atol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["0", "1"])
def test_sourceshape_tile_kernels_many_tiles(gpu, orc, tmp_path, kernel):
    """Both tile kernels (0: FP64 FMAs, 1: FP64 tensor path; chosen once per process by LAPH_SOURCESHAPE_KERNEL)
    on L = 20: 1000 sites per parity class, 32 site tiles with a ragged last one, off-diagonal tile pairs."""
    L, nev = 20, 16
    rng = np.random.default_rng(20)
    V, _ = np.linalg.qr(rng.normal(size=(3 * L ** 3, nev)) + 1j * rng.normal(size=(3 * L ** 3, nev)))
    np.save(tmp_path / "V.npy", V)
    script = ("import sys, numpy as np, laph_eigsys_b200 as lb; "
              "np.save(sys.argv[2], lb.sourceshape(np.load(sys.argv[1]), int(sys.argv[3])))")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    subprocess.run([sys.executable, "-c", script, str(tmp_path / "V.npy"), str(tmp_path / "psi.npy"), str(L)],
                   env=dict(os.environ, LAPH_SOURCESHAPE_KERNEL=kernel), cwd=root, check=True, timeout=300)
    psi = np.load(tmp_path / "psi.npy")
    ref = orc.sourceshape(V, L)
    assert np.abs(psi - ref).max() <= 1e-12 * np.abs(ref).max()


def test_sourceshape_rejects_odd_L():
    with pytest.raises(lb.LaphError) as e:
        lb.sourceshape_avg(5, np.ones(27))
    assert e.value.status == lb._lib.LAPH_EINVAL


def test_ascii_writer_matches_ostream_setprecision_12(tmp_path):
    """write_sourceshape_ascii formats with std::ostream << setprecision(12) (modules/read_write.cpp:205-220);
    the library's %.12g writer must give the same bytes, exponents and trailing-zero trimming included."""
    vals = [0.0, 2.0, 2.8284271247461903, 1e-5, 123456789012.5, 1.5e-300, 7.0e20, 0.1, 3.4641016151377544,
            12.000000000000002]
    r = np.array(vals)
    psi = np.array(vals[::-1])
    lb.write_sourceshape(tmp_path, 7, 3, 11, r, psi)
    got = open(tmp_path / "sourceshape_nev11.7.3").read()
    src = tmp_path / "fmt.cpp"
    src.write_text(
        "#include <fstream>\n#include <iomanip>\n#include <iostream>\nint main(){double a;double b;\n"
        "std::cout << \"#r\\tpsi(r)\" << std::endl;\n"
        "while (std::cin >> a >> b) std::cout << std::setprecision(12) << a << \" \" << b << std::endl;}\n")
    exe = tmp_path / "fmt"
    subprocess.run(["g++", "-O1", "-o", str(exe), str(src)], check=True, timeout=120)
    feed = "".join(f"{float(a)!r} {float(b)!r}\n" for a, b in zip(r, psi))
    want = subprocess.run([str(exe)], input=feed, capture_output=True, text=True, check=True).stdout
    assert got == want
