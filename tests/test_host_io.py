"""Host-side product logic on CPU: LIME/ILDG I/O against the oracle restatement
of read_lime_gauge_field_doubleprec_timeslices, eigensystem files and
check_trace, parameters.txt quirks, recover_spectrum / fix_phase."""
import os
import struct

import numpy as np
import pytest

import laph_eigsys_b200 as lb
from laph_eigsys_b200 import _lib


def test_lime_roundtrip_matches_oracle_reader(tmp_path, orc):
    L, T = 4, 6
    conf = lb.gauge_random(L, T, 0.4, 1227)
    p = tmp_path / "conf.1227"
    lb.lime_write_gauge(p, conf, L, T)
    assert os.path.getsize(p) > T * L ** 3 * 72 * 8
    got = lb.lime_read_gauge(p, T, L, 0, T - 1)
    assert np.array_equal(got, conf)
    sub = lb.lime_read_gauge(p, T, L, 2, 4)
    st, ref = orc.lime_read_gauge(p, T, L, 2, 4)
    assert st == 0
    assert np.array_equal(sub, ref) and np.array_equal(sub, conf[2:5])
    # map_timeslice_to_eigen == spatial slots 1..3
    assert np.array_equal(orc.map_timeslice(conf[3], L), lb.spatial_links(conf[3]))


def test_lime_file_layout_is_big_endian_ildg(tmp_path):
    L, T = 3, 2
    conf = lb.gauge_random(L, T, 0.4, 5)
    p = tmp_path / "c"
    lb.lime_write_gauge(p, conf, L, T)
    raw = open(p, "rb").read()
    assert raw[:4] == bytes([0x45, 0x67, 0x89, 0xab])
    # locate the binary record: header magic + type
    i = raw.index(b"ildg-binary-data") - 16
    n = struct.unpack(">Q", raw[i + 8:i + 16])[0]
    assert n == L ** 3 * T * 72 * 8
    data = raw[i + 144:i + 144 + n]
    # first site (t=0,z=0,y=0,x=0), mu=x first -> conf slot 1, element (0,0)
    re0, im0 = struct.unpack(">dd", data[:16])
    assert re0 == conf[0, 0, 1, 0, 0].real and im0 == conf[0, 0, 1, 0, 0].imag
    # second site in file order is x=1 -> site index 1*L*L
    re1 = struct.unpack(">d", data[72 * 8:72 * 8 + 8])[0]
    assert re1 == conf[0, L * L, 1, 0, 0].real


def _lime_record(typ, payload, mb=True, me=True):
    h = bytearray(144)
    h[0:4] = bytes([0x45, 0x67, 0x89, 0xab])
    h[4:6] = (1).to_bytes(2, "big")
    h[6:8] = ((0x8000 if mb else 0) | (0x4000 if me else 0)).to_bytes(2, "big")
    h[8:16] = len(payload).to_bytes(8, "big")
    h[16:16 + len(typ)] = typ.encode()
    pad = (-len(payload)) % 8
    return bytes(h) + payload + b"\0" * pad


@pytest.mark.parametrize("case,status,ref_status", [
    ("missing", _lib.LAPH_EIO, 500),
    ("norecord", _lib.LAPH_ENORECORD, -2),
    ("badsize", _lib.LAPH_ESIZE, 501),
    ("single", _lib.LAPH_ESINGLE, 502),
    ("truncated", _lib.LAPH_EIO, 500),
])
def test_lime_error_paths(tmp_path, orc, case, status, ref_status):
    L, T = 3, 2
    p = tmp_path / "bad"
    full = L ** 3 * T * 72 * 8
    if case == "norecord":
        p.write_bytes(_lime_record("ildg-format", b"<xml/>"))
    elif case == "badsize":
        p.write_bytes(_lime_record("ildg-binary-data", b"\0" * 800))
    elif case == "single":
        p.write_bytes(_lime_record("ildg-binary-data", b"\0" * (full // 2)))
    elif case == "truncated":
        rec = _lime_record("ildg-binary-data", b"\0" * full)
        p.write_bytes(rec[:144 + full // 3])
    with pytest.raises(lb.LaphError) as e:
        lb.lime_read_gauge(p, T, L, 0, T - 1)
    assert e.value.status == status
    st, _ = orc.lime_read_gauge(p, T, L, 0, T - 1)
    assert st == ref_status


def test_eigsys_files_and_check_trace(tmp_path):
    rng = np.random.default_rng(0)
    dim, nev = 96, 7
    A = rng.normal(size=(dim, nev)) + 1j * rng.normal(size=(dim, nev))
    Q, _ = np.linalg.qr(A)
    Q = np.asfortranarray(Q)
    ok, tr, sm = lb.check_trace(Q)
    VdV = Q.conj().T @ Q
    assert abs(tr - np.trace(VdV).real) < 1e-12 and abs(sm - VdV.sum().real) < 1e-12
    lb.write_eigsys_bin(tmp_path, "eigenvectors", 1227, 5, Q)
    raw = open(tmp_path / "eigenvectors.1227.005", "rb").read()
    assert raw == Q.tobytes(order="F")
    assert np.array_equal(lb.read_eigsys_bin(tmp_path, "eigenvectors", 1227, 5, dim, nev), Q)
    ev = np.linspace(-1, 0, nev)
    lb.write_eigenvalues_bin(tmp_path, "eigenvalues", 1227, 5, ev)
    assert open(tmp_path / "eigenvalues.1227.005", "rb").read() == ev.tobytes()
    # damaged eigenvectors: nothing is written (the reference exits)
    bad = Q * 1.01
    with pytest.raises(lb.LaphError) as e:
        lb.write_eigsys_bin(tmp_path, "eigenvectors", 1227, 6, bad)
    assert e.value.status == _lib.LAPH_ETRACE
    assert not (tmp_path / "eigenvectors.1227.006").exists()


def test_parameters_parser_quirks(tmp_path):
    p = tmp_path / "parameters.txt"
    p.write_text("# comment\nconfig_path = /gauges\nLT = 48\nLX = 24\nNEV = 120\nalpha_1 = 0.62\n"
                 "alpha_2 = 0.52\niter = 3\nLAM_L = 11.8\nLAM_C = 0.6\nDEG = 8\nOMP_THRDS = 2\n"
                 "alpha_1_i = 0.4\nalpha_1_f = 0.7\nalpha_2_i = 0.3\nalpha_2_f = 0.6\nautotune = 4\nfilter_deg = 56\n"
                 "LT=99\nsmear = stout\nDEG = 12")  # unterminated last line is dropped
    c = lb.parse_parameters(p)
    assert c["config_path"] == "/gauges" and c["LT"] == 48 and c["LX"] == 24 and c["NEV"] == 120
    assert c["DEG"] == 8 and c["iter"] == 3 and abs(c["LAM_L"] - 11.8) < 1e-15
    assert c["V3"] == 24 ** 3 and c["MAT_ENTRIES"] == 3 * 24 ** 3 and c["V_TS"] == 72 * 24 ** 3
    assert c["smear"] == lb.SMEAR_STOUT
    assert (c["alpha_1_i"], c["alpha_1_f"], c["alpha_2_i"], c["alpha_2_f"]) == (0.4, 0.7, 0.3, 0.6)
    assert c["autotune"] == 4 and c["filter_deg"] == 56
    p.write_text("LT = 4\n\nLX = 4\n")
    with pytest.raises(lb.LaphError) as e:
        lb.parse_parameters(p)
    assert e.value.status == _lib.LAPH_EPARSE


def test_recover_spectrum_and_fix_phase(orc):
    theta = np.array([50.0, 3.0, 1.2, 1.0])
    assert np.allclose(lb.recover_spectrum(theta, 8, 11.8, 0.6), orc.recover_spectrum(theta, 8, 11.8, 0.6),
                       rtol=0, atol=1e-15)
    rng = np.random.default_rng(1)
    V = rng.normal(size=(30, 4)) + 1j * rng.normal(size=(30, 4))
    a, pa = lb.fix_phase(V)
    b, pb = orc.fix_phase(V)
    assert np.abs(a - b).max() < 1e-15 and np.array_equal(pa, pb)


def test_gauge_random_deterministic_and_seeded():
    a = lb.gauge_random(3, 2, 0.3, 11)
    b = lb.gauge_random(3, 2, 0.3, 11)
    c = lb.gauge_random(3, 2, 0.3, 12)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    # eps = 0 gives the unit field
    u = lb.gauge_random(3, 1, 0.0, 1)
    assert np.abs(u - np.eye(3)).max() < 1e-14


def test_lime_fp32_roundtrip_and_info(tmp_path):
    """FP32 ILDG files (the reference stops at them, io.cpp:72-79): written big-endian with an ildg-format record,
    read back widened to FP64 equal to the FP32-rounded links; the strict reader keeps the reference's error."""
    L, T = 4, 3
    conf = lb.gauge_random(L, T, 0.3, 1234)
    p32, p64 = tmp_path / "c32", tmp_path / "c64"
    lb.lime_write_gauge(p32, conf, L, T, precision=32)
    lb.lime_write_gauge(p64, conf, L, T)
    assert lb.lime_info(p32) == (L, L, L, T, 32)
    assert lb.lime_info(p64) == (L, L, L, T, 64)
    got, prec = lb.lime_read_gauge_any(p32, T, L, 1, 2)
    assert prec == 32
    want = conf[1:3].real.astype(np.float32).astype(np.float64) + 1j * conf[1:3].imag.astype(np.float32)
    assert np.array_equal(got, want)
    got64, prec64 = lb.lime_read_gauge_any(p64, T, L, 0, T - 1)
    assert prec64 == 64 and np.array_equal(got64, conf)
    with pytest.raises(lb.LaphError) as e:
        lb.lime_read_gauge(p32, T, L, 0, 0)
    assert e.value.status == _lib.LAPH_ESINGLE
    # the record sizes of an FP32 file: 144 + xml (padded) + 144 + V3 T 72 4
    raw = open(p32, "rb").read()
    assert len(raw) % 8 == 0 and len(raw) > L ** 3 * T * 72 * 4


def test_lime_precision_mismatch_and_missing_format(tmp_path):
    L, T = 3, 2
    n64 = L ** 3 * T * 72 * 8
    xml = ("<?xml version=\"1.0\"?><ildgFormat><precision>32</precision><lx>3</lx><ly>3</ly><lz>3</lz>"
           "<lt>2</lt></ildgFormat>").encode()
    p = tmp_path / "mismatch"
    p.write_bytes(_lime_record("ildg-format", xml, me=False) + _lime_record("ildg-binary-data", b"\0" * n64,
                                                                          mb=False))
    with pytest.raises(lb.LaphError) as e:
        lb.lime_read_gauge_any(p, T, L, 0, 0)
    assert e.value.status == _lib.LAPH_ESIZE
    with pytest.raises(lb.LaphError) as e:
        lb.lime_info(p)
    assert e.value.status == _lib.LAPH_ESIZE
    # the strict reader ignores the XML, as the reference does
    conf = lb.lime_read_gauge(p, T, L, 0, 0)
    assert np.all(conf == 0)
    q = tmp_path / "noformat"
    q.write_bytes(_lime_record("ildg-binary-data", b"\0" * (n64 // 2)))
    with pytest.raises(lb.LaphError) as e:
        lb.lime_info(q)
    assert e.value.status == _lib.LAPH_ENORECORD
    got, prec = lb.lime_read_gauge_any(q, T, L, 0, T - 1)
    assert prec == 32 and np.all(got == 0)
    r = tmp_path / "badsize"
    r.write_bytes(_lime_record("ildg-binary-data", b"\0" * 800))
    with pytest.raises(lb.LaphError) as e:
        lb.lime_read_gauge_any(r, T, L, 0, 0)
    assert e.value.status == _lib.LAPH_ESIZE


def test_reset_phase_matches_oracle_and_is_overridden_by_fix_phase(orc):
    """reset_phase rotates each column's first entry to the wanted phase; ev_ts then calls fix_phase on the
    original block (src/ev_ts.cpp:304-312), so the written vectors are those of fix_phase alone."""
    rng = np.random.default_rng(7)
    V = rng.normal(size=(48, 5)) + 1j * rng.normal(size=(48, 5))
    want = rng.uniform(-np.pi, np.pi, 5)
    Vr = lb.reset_phase(V, want)
    assert np.abs(Vr - orc.reset_phase(V, want)).max() < 1e-15
    assert np.abs(np.angle(Vr[0]) - want).max() < 1e-13
    assert np.allclose(np.abs(Vr), np.abs(V), rtol=0, atol=1e-15)
    Vf, ph = lb.fix_phase(V)
    assert np.abs(lb.reset_phase(V, ph) - V).max() < 1e-14  # the block's own phases: no change
    assert np.abs(lb.reset_phase(V, np.zeros(5)) - Vf).max() < 1e-14  # phase 0 is fix_phase
    assert lb.lib.laph_reset_phase_host(0, 1, None, None, None) == _lib.LAPH_EINVAL
    assert lb.lib.laph_reset_phase_host(48, 1, None, None, None) == _lib.LAPH_EINVAL


def test_read_eigenvalues_ascii(tmp_path):
    ev = -np.sort(np.random.default_rng(3).uniform(0, 2, 7))
    pre = tmp_path / "eigenvalues"
    # timeslice first, then configuration; any whitespace between values
    (tmp_path / "eigenvalues.005.1227").write_text("  ".join(repr(float(v)) for v in ev[:3]) + "\n"
                                                    + "\n".join(repr(float(v)) for v in ev[3:]) + "\n")
    assert np.array_equal(lb.read_eigenvalues_ascii(pre, 1227, 5, 7), ev)
    assert np.array_equal(lb.read_eigenvalues_ascii(pre, 1227, 5, 4), ev[:4])
    with pytest.raises(lb.LaphError) as e:
        lb.read_eigenvalues_ascii(pre, 1227, 5, 8)
    assert e.value.status == _lib.LAPH_ESIZE
    with pytest.raises(lb.LaphError) as e:
        lb.read_eigenvalues_ascii(pre, 1227, 6, 7)
    assert e.value.status == _lib.LAPH_EIO


def test_gauge_matrices_file_is_raw_eigen_matrix3cd(tmp_path):
    G = lb.gauge_random(3, 1, 0.5, 21)[0, :, 0]  # 27 SU(3) matrices, row-major (a, b)
    p = tmp_path / "gauge_trafo.bin"
    lb.write_gauge_matrices(p, G)
    raw = np.fromfile(p, dtype=np.complex128).reshape(27, 9)
    assert raw.nbytes == 27 * 144
    # Eigen memory order is column-major: entry (a, b) at 3 b + a
    assert all(raw[v, 3 * b + a] == G[v, a, b] for v in (0, 13, 26) for a in range(3) for b in range(3))
    assert np.array_equal(lb.read_gauge_matrices(p, 27), G)
    with pytest.raises(lb.LaphError) as e:
        lb.read_gauge_matrices(p, 28)
    assert e.value.status == _lib.LAPH_ESIZE
    with pytest.raises(lb.LaphError) as e:
        lb.read_gauge_matrices(tmp_path / "missing", 27)
    assert e.value.status == _lib.LAPH_EIO


_STATUS_OF_REF = {0: _lib.LAPH_OK, 500: _lib.LAPH_EIO, 501: _lib.LAPH_ESIZE, 502: _lib.LAPH_ESINGLE,
                  -2: _lib.LAPH_ENORECORD}


def test_lime_reader_fuzz_matches_reference_restatement(tmp_path, orc):
    """Mutated LIME files (truncations, corrupted header bytes, wrong lengths, extra records before or after the
    binary one, a second binary record): laph_lime_read_gauge ends with the status the reference's reader ends
    with (read_lime_gauge_field_doubleprec_timeslices, restated by the oracle: exit codes 500/501/502/-2) and, when
    both succeed, with the same links, for random timeslice ranges."""
    L, T = 3, 3
    conf = lb.gauge_random(L, T, 0.4, 99)
    good = tmp_path / "good"
    lb.lime_write_gauge(good, conf, L, T)
    base = good.read_bytes()
    i_bin = base.index(b"ildg-binary-data") - 16
    n_pay = L ** 3 * T * 72 * 8
    rng = np.random.default_rng(7)
    p = tmp_path / "mutant"
    seen = set()
    for case in range(400):
        kind = int(rng.integers(0, 7))
        b = bytearray(base)
        if kind == 0:    # truncated anywhere
            b = b[:int(rng.integers(0, len(b)))]
        elif kind == 1:  # one byte of a record header changed
            hdr = int(rng.choice([0, i_bin]))
            k = int(rng.integers(0, 40))
            b[hdr + k] ^= int(rng.integers(1, 256))
        elif kind == 2:  # binary record length off by a little, halved or doubled
            n = int(rng.choice([n_pay - 8, n_pay + 8, n_pay // 2, 2 * n_pay, n_pay - 1]))
            b[i_bin + 8:i_bin + 16] = n.to_bytes(8, "big")
        elif kind == 3:  # an extra record of another type first
            junk = bytes(rng.integers(0, 256, int(rng.integers(0, 40)), dtype=np.uint8))
            b = bytearray(_lime_record("xlf-info", junk, me=False)) + b
        elif kind == 4:  # junk after the last record
            b = b + bytes(rng.integers(0, 256, int(rng.integers(1, 300)), dtype=np.uint8))
        elif kind == 5:  # a second, different binary record after the first: the first one counts
            other = bytes(rng.integers(0, 256, n_pay, dtype=np.uint8))
            b = b + bytearray(_lime_record("ildg-binary-data", other, mb=False))
        else:            # a binary record of the right size but only part of its payload present
            b = b[:i_bin + 144 + int(rng.integers(0, n_pay))]
        p.write_bytes(bytes(b))
        t0 = int(rng.integers(0, T))
        t1 = int(rng.integers(t0, T))
        st_ref, ref = orc.lime_read_gauge(p, T, L, t0, t1)
        want = _STATUS_OF_REF[st_ref]
        try:
            got = lb.lime_read_gauge(p, T, L, t0, t1)
            st = _lib.LAPH_OK
        except lb.LaphError as e:
            st = e.status
        assert st == want, (case, kind, st, st_ref)
        if st == _lib.LAPH_OK:
            assert np.array_equal(got, ref), (case, kind)
        seen.add((kind, st))
    assert {s for _, s in seen} >= {_lib.LAPH_OK, _lib.LAPH_EIO, _lib.LAPH_ESIZE, _lib.LAPH_ESINGLE,
                                    _lib.LAPH_ENORECORD}


def test_ildg_format_record_fuzz_never_crashes(tmp_path):
    """Random and truncated ildg-format payloads in front of a valid FP64 record: lime_info and the any-precision
    reader return a status (never crash or hang); wherever the XML declares nothing contradicting the data, the
    links come back exactly."""
    L, T = 3, 2
    conf = lb.gauge_random(L, T, 0.4, 5)
    n64 = L ** 3 * T * 72 * 8
    payload = bytearray(n64)
    good = tmp_path / "g"
    lb.lime_write_gauge(good, conf, L, T)
    raw = good.read_bytes()
    data = raw[raw.index(b"ildg-binary-data") - 16:]
    rng = np.random.default_rng(11)
    tags = [b"<precision>", b"</precision>", b"<lx>", b"<lt>", b"64", b"32", b"3", b"2", b"<", b">", b"\0", b"x"]
    p = tmp_path / "f"
    ok = 0
    for case in range(300):
        xml = b"".join(rng.choice(tags, size=int(rng.integers(0, 30))))
        if rng.random() < 0.3:
            xml = bytes(rng.integers(0, 256, int(rng.integers(0, 200)), dtype=np.uint8))
        p.write_bytes(_lime_record("ildg-format", xml, me=False) + data)
        try:
            lb.lime_info(p)
        except lb.LaphError as e:
            assert e.status in (_lib.LAPH_ESIZE, _lib.LAPH_ENORECORD, _lib.LAPH_EIO, _lib.LAPH_EPARSE)
        try:
            got, prec = lb.lime_read_gauge_any(p, T, L, 0, T - 1)
        except lb.LaphError as e:
            assert e.status == _lib.LAPH_ESIZE  # the XML declared 32-bit reals over FP64 data
            continue
        assert prec == 64 and np.array_equal(got, conf)
        ok += 1
    assert ok > 100


def test_lime_reorder_transcribes_reference_loop(tmp_path, orc):
    """read_lime_gauge_field_doubleprec_timeslices' copy loop (modules/io.cpp:84-131), transcribed: file order
    t, z, y, x with 72 big-endian doubles per site in ILDG mu order x, y, z, t; config position
    ((t - t_i) LX LY LZ + x LY LZ + y LZ + z) 72, U_x..U_z to slots 1..3 and U_t to slot 0, each 3x3 row-major
    complex.  Random (not SU(3)) payload, so every number's place is checked."""
    L, T, ti, tf = 3, 4, 1, 2
    rng = np.random.default_rng(5)
    vals = rng.normal(size=L ** 3 * T * 72)
    p = tmp_path / "conf"
    p.write_bytes(_lime_record("ildg-binary-data", vals.astype(">f8").tobytes()))
    filec = (vals[0::2] + 1j * vals[1::2]).reshape(T, L, L, L, 4, 3, 3)  # [t][z][y][x][mu_file][i][j]
    want = np.transpose(filec, (0, 3, 2, 1, 4, 5, 6)).reshape(T, L ** 3, 4, 3, 3)[:, :, [3, 0, 1, 2]][ti:tf + 1]
    assert np.array_equal(lb.lime_read_gauge(p, T, L, ti, tf), want)
    st, ref = orc.lime_read_gauge(p, T, L, ti, tf)
    assert st == 0 and np.array_equal(ref, want)


def test_reference_quirks_of_the_small_host_functions(orc):
    """check_trace is one-sided as in read_write.cpp:29-33 (|tr| - nev > eps fails, a shrunken block passes);
    recover_spectrum gives NaN for theta < 1 (acosh, recover_spec.cpp:24-30), where the eigenvalue lies above
    LAM_C; fix_phase leaves a column whose first entry is 0 as it is (arg 0 = 0)."""
    rng = np.random.default_rng(9)
    Q, _ = np.linalg.qr(rng.normal(size=(60, 5)) + 1j * rng.normal(size=(60, 5)))
    assert lb.check_trace(Q)[0]
    assert lb.check_trace(Q * 0.99)[0]          # trace 4.9 < nev: passes, as in the reference
    assert not lb.check_trace(Q * 1.0001)[0]    # trace above nev by more than 1e-9: fails
    th = np.array([3.0, 1.0, 0.5])
    a = lb.recover_spectrum(th, 8, 12.0, 0.6)
    b = orc.recover_spectrum(th, 8, 12.0, 0.6)
    assert np.isnan(a[2]) and np.isnan(b[2]) and abs(a[1] + 0.6) < 1e-15 and np.allclose(a[:2], b[:2], rtol=0,
                                                                                          atol=1e-15)
    V = Q.copy()
    V[0, 2] = 0.0
    Vf, ph = lb.fix_phase(V)
    assert ph[2] == 0.0 and np.array_equal(Vf[:, 2], V[:, 2])


def test_fp32_reader_refuses_truncated_record(tmp_path):
    """The any-precision reader applies the same whole-record rule to FP32 files."""
    L, T = 3, 3
    conf = lb.gauge_random(L, T, 0.3, 8)
    p = tmp_path / "c32"
    lb.lime_write_gauge(p, conf, L, T, precision=32)
    raw = p.read_bytes()
    p.write_bytes(raw[:len(raw) - 100])
    with pytest.raises(lb.LaphError) as e:
        lb.lime_read_gauge_any(p, T, L, 0, 0)  # the first timeslice is all there, the record is not
    assert e.value.status == _lib.LAPH_EIO


def test_recover_spectrum_transcribes_reference():
    """invert_Tn then invert_B (modules/recover_spec.cpp:13-30, applied in recover_spectrum :45-54):
    b = cosh(acosh(theta) / DEG), lambda_stored = (LAM_L - LAM_C) (b - 1) / 2 - LAM_C."""
    theta = np.array([1e6, 123.4, 2.5, 1.0 + 1e-9])
    for deg, lam_l, lam_c in ((8, 11.8, 0.6), (12, 12.0, 0.65), (3, 10.0, 1.5)):
        b = np.cosh(np.arccosh(theta) / deg)
        want = (lam_l - lam_c) * (b - 1) * 0.5 - lam_c
        got = lb.recover_spectrum(theta, deg, lam_l, lam_c)
        assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
