"""Pins against the reference's own code: oracle/_ref/ref_dump is built from the
reference's modules/par_io.cpp and modules/navigation.cpp (the parts of the path
that compile without Eigen, PETSc, SLEPc and c-lime).  laph_parse_parameters must
read every parameters.txt the way IO::set_values does, quirks included, and the
oracle's site indexing must use the reference's Nav lookup tables."""
import json
import os
import subprocess

import numpy as np
import pytest

import laph_eigsys_b200 as lb
from laph_eigsys_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "ref_dump")

pytestmark = pytest.mark.skipif(not os.path.isfile(REF), reason="oracle/_ref/ref_dump not built (no reference here)")


def ref(mode, path):
    r = subprocess.run([REF, mode, str(path)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout)


FULL = ("# LapH parameters\nconfig_path = /gauges/A40\nresult_path = /out\nin_path = /in\nphase_path = /ph\n"
        "LT = 48\nLX = 24\nNEV = 120\nalpha_1 = 0.62\nalpha_2 = 0.52\nalpha_1_i = 0.4\nalpha_1_f = 0.75\n"
        "alpha_2_i = 0.3\nalpha_2_f = 0.65\niter = 3\nLAM_L = 11.8\nLAM_C = 0.6\nDEG = 8\nOMP_THRDS = 4\n")

CASES = {
    "full": FULL,
    "unterminated_last_line": FULL + "DEG = 12",
    "no_space_around_equals": FULL + "LT=99\nNEV=7\n",
    "duplicate_keys_last_wins": FULL + "LX = 16\nLAM_C = 0.75\n",
    "extra_space_in_key": FULL.replace("DEG = 8", "DEG  = 8"),
    "line_without_equals": FULL + "just some words\n",
    "trailing_space_value": FULL + "iter = \n",
    "crlf": FULL.replace("\n", "\r\n"),
    "exponents_and_signs": FULL + "LAM_C = 6e-1\nalpha_1 = +0.5\nNEV = 0120\n",
    "missing_keys": "LT = 8\nLX = 4\n",
    "comment_not_first_char": FULL + " # not a comment = 5\n",
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_parser_matches_reference(tmp_path, name):
    p = tmp_path / "parameters.txt"
    p.write_bytes(CASES[name].encode())
    r = ref("params", p)
    assert not r["threw"]
    c = lb.parse_parameters(p)
    for k in ("LT", "LX", "NEV", "iter", "DEG", "OMP_THRDS", "V3", "MAT_ENTRIES", "V_TS"):
        assert c[k] == r[k], k
    for k, rk in (("alpha_1", "alpha_1"), ("alpha_2", "alpha_2"), ("alpha_1_i", "alpha_1_i"),
                  ("alpha_1_f", "alpha_1_f"), ("alpha_2_i", "alpha_2_i"), ("alpha_2_f", "alpha_2_f"),
                  ("LAM_L", "lambda_l"), ("LAM_C", "lambda_c")):
        assert c[k] == r[rk], k
    for k, rk in (("config_path", "conf"), ("result_path", "res"), ("in_path", "in_path"),
                  ("phase_path", "phase_path")):
        assert c[k] == r[rk], k


@pytest.mark.parametrize("text", ["LT = 4\n\nLX = 4\n", "LT = 4\nLX =\n", FULL + "NEV = 1\n\n"])
def test_parser_errors_where_reference_throws(tmp_path, text):
    p = tmp_path / "parameters.txt"
    p.write_text(text)
    assert ref("params", p)["threw"]
    with pytest.raises(lb.LaphError) as e:
        lb.parse_parameters(p)
    assert e.value.status == _lib.LAPH_EPARSE


@pytest.mark.parametrize("L", [3, 4, 6])
def test_oracle_indexing_uses_reference_lookup_tables(tmp_path, orc, L):
    """Site i = x L^2 + y L + z with periodic neighbours (Nav::init): the oracle's assembled -Delta with unit links
    has -1 exactly at (3i + a, 3 up(i, mu) + a) and (3i + a, 3 dn(i, mu) + a), 6 on the diagonal."""
    p = tmp_path / "parameters.txt"
    p.write_text(f"LT = 4\nLX = {L}\nNEV = 4\n")
    nav = ref("nav", p)
    up, dn = np.array(nav["up"]), np.array(nav["dn"])
    V3 = L ** 3
    x, y, z = np.meshgrid(np.arange(L), np.arange(L), np.arange(L), indexing="ij")
    idx = lambda a, b, c: ((a % L) * L * L + (b % L) * L + (c % L)).ravel()  # noqa: E731
    assert np.array_equal(up[:, 0], idx(x + 1, y, z)) and np.array_equal(dn[:, 0], idx(x - 1, y, z))
    assert np.array_equal(up[:, 1], idx(x, y + 1, z)) and np.array_equal(dn[:, 1], idx(x, y - 1, z))
    assert np.array_equal(up[:, 2], idx(x, y, z + 1)) and np.array_equal(dn[:, 2], idx(x, y, z - 1))
    U = np.zeros((V3, 3, 3, 3), dtype=np.complex128)
    U[:, :] = np.eye(3)
    A = orc.neglap_dense(U, L)
    B = np.zeros((3 * V3, 3 * V3))
    for i in range(V3):
        for a in range(3):
            B[3 * i + a, 3 * i + a] += 6.0
            for mu in range(3):
                B[3 * i + a, 3 * up[i, mu] + a] -= 1.0
                B[3 * i + a, 3 * dn[i, mu] + a] -= 1.0
    assert np.array_equal(A.real, B) and not np.any(A.imag)


KEYS_INT = ["LT", "LX", "NEV", "iter", "DEG", "OMP_THRDS"]
KEYS_FLOAT = ["alpha_1", "alpha_2", "alpha_1_i", "alpha_1_f", "alpha_2_i", "alpha_2_f", "LAM_L", "LAM_C"]
KEYS_PATH = ["config_path", "result_path", "in_path", "phase_path"]


def _random_file(rng):
    lines = []
    for _ in range(int(rng.integers(1, 25))):
        kind = rng.integers(0, 10)
        if kind == 0:
            lines.append("#" + "".join(rng.choice(list("abc =#"), size=int(rng.integers(0, 8)))))
            continue
        if kind == 1:
            lines.append("".join(rng.choice(list("xyz #-"), size=int(rng.integers(1, 8)))))  # no '='
            continue
        if kind == 2 and rng.random() < 0.15:
            lines.append("")  # the reference throws on an empty line
            continue
        pool = rng.integers(0, 4)
        if pool == 0:
            key = str(rng.choice(KEYS_INT))
            val = str(rng.choice(["8", "24", "0120", "-3", "+7", "12abc", "", " 5", "3.9"]))
        elif pool == 1:
            key = str(rng.choice(KEYS_FLOAT))
            val = str(rng.choice(["0.62", "6e-1", "+0.5", "-1.25e+1", "11.8", "", "1e", "nan", ".5"]))
        elif pool == 2:
            key = str(rng.choice(KEYS_PATH))
            val = "/" + "".join(rng.choice(list("abc/_ =.-"), size=int(rng.integers(0, 12))))
        else:
            key = str(rng.choice(["LY", "ev_path_1", "lambda_l", "foo", "Lx", "NEV2"]))
            val = "1"
        sep = str(rng.choice([" = ", "=", " =", "= ", "  = ", " =  "]))
        pre = " " if rng.random() < 0.05 else ""
        lines.append(pre + key + sep + val)
    eol = "\r\n" if rng.random() < 0.1 else "\n"
    text = eol.join(lines)
    if rng.random() < 0.8:
        text += eol
    return text


def test_parser_fuzz_against_reference(tmp_path):
    rng = np.random.default_rng(2024)
    p = tmp_path / "parameters.txt"
    threw = 0
    for case in range(300):
        text = _random_file(rng)
        p.write_bytes(text.encode())
        r = ref("params", p)
        if r["threw"]:
            threw += 1
            with pytest.raises(lb.LaphError) as e:
                lb.parse_parameters(p)
            assert e.value.status == _lib.LAPH_EPARSE, text
            continue
        c = lb.parse_parameters(p)
        for k in KEYS_INT + ["V3", "MAT_ENTRIES", "V_TS"]:
            assert c[k] == r[k], (k, text)
        for k in KEYS_FLOAT:
            rk = {"LAM_L": "lambda_l", "LAM_C": "lambda_c"}.get(k, k)
            assert c[k] == r[rk] or (np.isnan(c[k]) and np.isnan(r[rk])), (k, text)
        for k, rk in zip(KEYS_PATH, ["conf", "res", "in_path", "phase_path"]):
            assert c[k] == r[rk], (k, text)
    assert 0 < threw < 300


@pytest.mark.parametrize("L", [4, 6])
def test_oracle_sourceshape_walks_reference_lookup_tables(tmp_path, orc, L):
    """source_shape_complete reaches x + r by r_i steps of Nav::get_up in x, then y, then z
    (get_vectorial_dst_ind, modules/sourceshape_funcs.cpp:9-24): psi(r) built here from the reference's own tables
    equals the oracle's (and with it the device kernel's, pinned to the oracle elsewhere)."""
    p = tmp_path / "parameters.txt"
    p.write_text(f"LT = 4\nLX = {L}\nNEV = 4\n")
    up = np.array(ref("nav", p)["up"])
    V3, nev = L ** 3, 5
    rng = np.random.default_rng(L)
    V, _ = np.linalg.qr(rng.normal(size=(3 * V3, nev)) + 1j * rng.normal(size=(3 * V3, nev)))
    blocks = V.reshape(V3, 3, nev)
    psi = []
    for r1 in range(0, L, 2):
        for r2 in range(0, L, 2):
            for r3 in range(0, L, 2):
                dst = np.arange(V3)
                for d, r in enumerate((r1, r2, r3)):
                    for _ in range(r):
                        dst = up[dst, d]
                M = np.einsum("xan,xbn->xab", blocks[dst], blocks.conj())
                psi.append(np.sqrt((np.abs(M) ** 2).sum(axis=(1, 2))).sum())
    ref_psi = np.array(psi)
    assert np.abs(orc.sourceshape(V, L) - ref_psi).max() <= 1e-12 * ref_psi.max()


@pytest.mark.parametrize("L", [3, 4])
def test_oracle_displacement_uses_reference_lookup_tables(tmp_path, orc, L):
    """right_displacement_one_dir (modules/config_utils.cpp:344-382) with the reference's iup / idown tables:
    W(x) = (U_dir(x) V(iup[x][dir]) - U_dir(idown[x][dir])^dag V(idown[x][dir])) / 2, against the oracle."""
    p = tmp_path / "parameters.txt"
    p.write_text(f"LT = 4\nLX = {L}\nNEV = 4\n")
    nav = ref("nav", p)
    up, dn = np.array(nav["up"]), np.array(nav["dn"])
    V3, nev = L ** 3, 3
    U = lb.gauge_random(L, 1, 0.5, 17)[0, :, 1:4]  # (V3, 3, 3, 3): [site][dir][a][b]
    rng = np.random.default_rng(3)
    V = rng.normal(size=(3 * V3, nev)) + 1j * rng.normal(size=(3 * V3, nev))
    blocks = V.reshape(V3, 3, nev)
    for d in range(3):
        fw = np.einsum("xab,xbn->xan", U[:, d], blocks[up[:, d]])
        bw = np.einsum("xba,xbn->xan", U[dn[:, d], d].conj(), blocks[dn[:, d]])
        W = (0.5 * (fw - bw)).reshape(3 * V3, nev)
        assert np.abs(orc.displace(U, L, d, V) - W).max() <= 1e-14 * np.abs(W).max()


@pytest.mark.parametrize("L", [3, 4])
def test_oracle_matvec_uses_reference_lookup_tables(tmp_path, orc, L):
    """tv2 (modules/shell_matop.cpp:16-103) with the reference's get_up / get_dn on random links:
    B x = c (sum_mu U_mu(k) x(up) + U_mu(dn)^dag x(dn) - 6 x(k)) + a x(k), c = 2 / (LAM_L - LAM_C),
    a = 1 + c LAM_C; tv_iter's T_deg(B) x by the three-term recurrence, against the oracle for deg 2, 3, 5."""
    p = tmp_path / "parameters.txt"
    p.write_text(f"LT = 4\nLX = {L}\nNEV = 4\n")
    nav = ref("nav", p)
    up, dn = np.array(nav["up"]), np.array(nav["dn"])
    V3 = L ** 3
    U = lb.gauge_random(L, 1, 0.5, 23)[0, :, 1:4]
    lam_l, lam_c = 11.8, 0.6
    c = 2.0 / (lam_l - lam_c)
    a = 1.0 + c * lam_c

    def B(v):
        x = v.reshape(V3, 3)
        hop = np.zeros_like(x)
        for mu in range(3):
            hop += np.einsum("kab,kb->ka", U[:, mu], x[up[:, mu]])
            hop += np.einsum("kba,kb->ka", U[dn[:, mu], mu].conj(), x[dn[:, mu]])
        return (c * (hop - 6.0 * x) + a * x).ravel()

    rng = np.random.default_rng(L)
    x = rng.normal(size=3 * V3) + 1j * rng.normal(size=3 * V3)
    t_prev, t_cur = x, B(x)
    for deg in range(2, 6):
        t_prev, t_cur = t_cur, 2.0 * B(t_cur) - t_prev
        if deg in (2, 3, 5):
            got = orc.tv_iter(U, L, lam_l, lam_c, deg, x)
            assert np.abs(got - t_cur).max() <= 1e-13 * np.abs(t_cur).max(), deg


def _proj_su3_imp(M):
    """proj_to_su3_imp (modules/timeslice.cpp:90-104): M ((M^dag M)^{1/2})^{-1}, then times det^{-1/3} with the
    principal complex cube root, for a stack of 3x3 matrices."""
    H = np.conj(np.swapaxes(M, -1, -2)) @ M
    w, Q = np.linalg.eigh(H)
    inv_sqrt = (Q * (1.0 / np.sqrt(w))[..., None, :]) @ np.conj(np.swapaxes(Q, -1, -2))
    W = M @ inv_sqrt
    return W * (1.0 / np.power(np.linalg.det(W).astype(complex), 1.0 / 3.0))[..., None, None]


@pytest.mark.parametrize("L", [3, 4])
def test_oracle_ape_uses_reference_lookup_tables(tmp_path, orc, L):
    """Tslice::smearing_ape (modules/timeslice.cpp:196-239) with the reference's get_up / get_dn, including its
    backward staple U[mu][nd]^dag U[mu][d] U[nu][d] (the quirk: U[nu][d] where U[nu][nd] is meant), two iterations,
    against the oracle in compat mode."""
    p = tmp_path / "parameters.txt"
    p.write_text(f"LT = 4\nLX = {L}\nNEV = 4\n")
    nav = ref("nav", p)
    up, dn = np.array(nav["up"]), np.array(nav["dn"])
    U = lb.gauge_random(L, 1, 0.4, 31)[0, :, 1:4].copy()
    alpha, iters = 0.5, 2
    dag = lambda m: np.conj(np.swapaxes(m, -1, -2))  # noqa: E731
    Us = U.copy()
    for _ in range(iters):
        new = np.empty_like(Us)
        for d in range(3):
            staple = np.zeros_like(Us[:, d])
            for nd in range(3):
                if nd == d:
                    continue
                mu = up[:, nd]
                nu = up[mu, d]
                eta = dn[nu, nd]
                staple += Us[:, nd] @ (Us[mu, d] @ dag(Us[eta, nd]))
                mu = dn[:, nd]
                nu = up[mu, d]
                staple += dag(Us[mu, nd]) @ (Us[mu, d] @ Us[nu, d])
            new[:, d] = Us[:, d] * (1.0 - alpha) + staple * (alpha / 4.0)
        Us = _proj_su3_imp(new)
    got = orc.smear_ape(U, L, alpha, iters, 1)
    assert np.abs(got - Us).max() <= 1e-12


@pytest.mark.parametrize("L", [3, 4])
def test_oracle_stout_uses_reference_lookup_tables(tmp_path, orc, L):
    """Tslice::smearing_stout (modules/timeslice.cpp:145-193) with the reference's get_up / get_dn and its
    backward-staple quirk: Omega = (rho / 4) C U^dag, q = (Omega^dag - Omega) / 2 - tr(Omega^dag - Omega) / 6,
    U' = exp(-q) U, two iterations, against the oracle in compat mode."""
    from scipy.linalg import expm
    p = tmp_path / "parameters.txt"
    p.write_text(f"LT = 4\nLX = {L}\nNEV = 4\n")
    nav = ref("nav", p)
    up, dn = np.array(nav["up"]), np.array(nav["dn"])
    U = lb.gauge_random(L, 1, 0.4, 37)[0, :, 1:4].copy()
    rho, iters = 0.1, 2
    dag = lambda m: np.conj(np.swapaxes(m, -1, -2))  # noqa: E731
    Us = U.copy()
    for _ in range(iters):
        new = np.empty_like(Us)
        for d in range(3):
            staple = np.zeros_like(Us[:, d])
            for nd in range(3):
                if nd == d:
                    continue
                mu = up[:, nd]
                nu = up[mu, d]
                eta = dn[nu, nd]
                staple += Us[:, nd] @ (Us[mu, d] @ dag(Us[eta, nd]))
                mu = dn[:, nd]
                nu = up[mu, d]
                staple += dag(Us[mu, nd]) @ (Us[mu, d] @ Us[nu, d])
            omega = (staple * (rho / 4.0)) @ dag(Us[:, d])
            A = dag(omega) - omega
            q = A * 0.5 - np.trace(A, axis1=1, axis2=2)[:, None, None] * np.eye(3) / 6.0
            new[:, d] = np.stack([expm(-qq) for qq in q]) @ Us[:, d]
        Us = new
    got = orc.smear_stout(U, L, rho, iters, 1)
    assert np.abs(got - Us).max() <= 1e-12


@pytest.mark.parametrize("L", [3, 4])
def test_oracle_hyp_uses_reference_lookup_tables(tmp_path, orc, L):
    """Tslice::smearing_hyp (modules/timeslice.cpp:243-369, get_dirs :106-122, decor :125-140) with the
    reference's get_up / get_dn: level 1 decorated links in slots dir / dir + 3 (perpendicular directions in
    get_dirs order), level 2 with plane = ((dir + 1) ^ (not_dir + 1)) - 1 and the decor storage map, two
    iterations, against the oracle."""
    p = tmp_path / "parameters.txt"
    p.write_text(f"LT = 4\nLX = {L}\nNEV = 4\n")
    nav = ref("nav", p)
    up, dn = np.array(nav["up"]), np.array(nav["dn"])
    U = lb.gauge_random(L, 1, 0.4, 41)[0, :, 1:4].copy()
    a1, a2, iters = 0.62, 0.52, 2
    dag = lambda m: np.conj(np.swapaxes(m, -1, -2))  # noqa: E731
    dirs = {0: (1, 2), 1: (0, 2), 2: (0, 1)}
    decor = {(0, 1): 0, (0, 2): 3, (1, 0): 1, (1, 2): 4, (2, 0): 2, (2, 1): 5}
    Us = U.copy()
    for _ in range(iters):
        dec = np.empty((Us.shape[0], 6, 3, 3), dtype=np.complex128)
        for d in range(3):
            for n_el, pd in enumerate(dirs[d]):
                inner = Us[:, pd] @ (Us[up[:, pd], d] @ dag(Us[up[:, d], pd]))
                m = dn[:, pd]
                inner = inner + dag(Us[m, pd]) @ (Us[m, d] @ Us[up[m, d], pd])
                dec[:, d + 3 * n_el] = _proj_su3_imp(Us[:, d] * (1 - a2) + inner * (a2 / 2.0))
        new = np.empty_like(Us)
        for d in range(3):
            outer = np.zeros_like(Us[:, d])
            for nd in range(3):
                if nd == d:
                    continue
                plane = ((d + 1) ^ (nd + 1)) - 1
                a, b = decor[(nd, plane)], decor[(d, plane)]
                mu = up[:, nd]
                eta = dn[up[mu, d], nd]
                outer += dec[:, a] @ (dec[mu, b] @ dag(dec[eta, a]))
                mu = dn[:, nd]
                outer += dag(dec[mu, a]) @ (dec[mu, b] @ dec[up[mu, d], a])
            new[:, d] = Us[:, d] * (1.0 - a1) + outer * (a1 / 4.0)
        Us = _proj_su3_imp(new)
    got = orc.smear_hyp(U, L, a1, a2, iters)
    assert np.abs(got - Us).max() <= 1e-12


def _refdir():
    """The reference checkout's directory as oracle/Makefile knows it ($LAPH_REFERENCE or the build machine's)."""
    try:
        out = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "refdir"], capture_output=True,
                             text=True, timeout=30)
        return out.stdout.strip()
    except Exception:
        return ""


REF_PARAMS = os.path.join(_refdir(), "src", "parameters.txt")


@pytest.mark.skipif(not os.path.isfile(REF_PARAMS), reason="the reference checkout is not on this machine")
def test_reference_shipped_parameters_file(tmp_path):
    """The parameters.txt the reference ships (src/parameters.txt, with its trailing spaces after values) parses
    to what IO::set_values stores (the command-line programs read their settings through this parser)."""
    p = tmp_path / "parameters.txt"
    p.write_bytes(open(REF_PARAMS, "rb").read())
    r = ref("params", p)
    assert not r["threw"]
    c = lb.parse_parameters(p)
    assert (c["LT"], c["LX"], c["NEV"], c["iter"], c["DEG"], c["OMP_THRDS"]) == (r["LT"], r["LX"], r["NEV"], r["iter"],
                                                                                 r["DEG"], r["OMP_THRDS"])
    for k, rk in (("alpha_1", "alpha_1"), ("alpha_2", "alpha_2"), ("alpha_1_i", "alpha_1_i"),
                  ("alpha_1_f", "alpha_1_f"),
                  ("alpha_2_i", "alpha_2_i"), ("alpha_2_f", "alpha_2_f"), ("LAM_L", "lambda_l"), ("LAM_C", "lambda_c")):
        assert c[k] == r[rk], k
    assert (c["config_path"], c["result_path"], c["in_path"]) == (r["conf"], r["res"], r["in_path"])


@pytest.mark.parametrize("L", [3, 4])
def test_oracle_plaquette_uses_reference_lookup_tables(tmp_path, orc, L):
    """plaque_timeslice / get_plaque_nx_ny (modules/config_utils.cpp:388-426) with the reference's iup / idown:
    the mean over sites and ordered direction pairs x != y of Re tr(U_x(i) U_y(i+x) U_x(i+y)^dag U_y(i)^dag) / 3
    (l = idown[iup[iup[i][x]][y]][x] = i + y), against the oracle."""
    p = tmp_path / "parameters.txt"
    p.write_text(f"LT = 4\nLX = {L}\nNEV = 4\n")
    nav = ref("nav", p)
    up, dn = np.array(nav["up"]), np.array(nav["dn"])
    U = lb.gauge_random(L, 1, 0.6, 53)[0, :, 1:4]
    dag = lambda m: np.conj(np.swapaxes(m, -1, -2))  # noqa: E731
    tot, cnt = 0.0, 0
    for x in range(3):
        for y in range(3):
            if x == y:
                continue
            j = up[:, x]
            k = up[j, y]
            l_ = dn[k, x]
            P = U[:, x] @ (U[j, y] @ (dag(U[l_, x]) @ dag(U[:, y])))
            tot += np.trace(P, axis1=1, axis2=2).real.sum() / 3.0
            cnt += L ** 3
    assert abs(orc.plaquette(U, L) - tot / cnt) < 1e-14


@pytest.mark.parametrize("L", [3, 4])
def test_oracle_assembled_operator_is_buildlaplacian(tmp_path, orc, L):
    """BuildLaplacian (modules/config_utils.cpp:18-58) with the reference's get_up / get_dn on random links:
    6 on the diagonal, -U_mu(i)(a, b) at (3i + a, 3 up + b), -U_mu(down)^dag(a, b) at (3i + a, 3 down + b), with
    its INSERT_VALUES (for L >= 3 no entry is set twice) -- the oracle's dense -Delta used by every spectrum test."""
    p = tmp_path / "parameters.txt"
    p.write_text(f"LT = 4\nLX = {L}\nNEV = 4\n")
    nav = ref("nav", p)
    up, dn = np.array(nav["up"]), np.array(nav["dn"])
    V3 = L ** 3
    U = lb.gauge_random(L, 1, 0.5, 59)[0, :, 1:4]
    A = np.zeros((3 * V3, 3 * V3), dtype=np.complex128)
    for i in range(V3):
        for c in range(3):
            A[3 * i + c, 3 * i + c] = 6.0
        for mu in range(3):
            u, d = up[i, mu], dn[i, mu]
            A[3 * i:3 * i + 3, 3 * u:3 * u + 3] = -U[i, mu]
            A[3 * i:3 * i + 3, 3 * d:3 * d + 3] = -U[d, mu].conj().T
    assert np.abs(orc.neglap_dense(U, L) - A).max() < 1e-15
