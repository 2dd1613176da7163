"""laph_eigsys_b200 -- B200 (sm_100a) implementation of the per-timeslice LapH
eigensystem path of HISKP-LQCD/LapH_EigSys.

The compute path is the CUDA library liblaph_gpu.so (C ABI: include/laph_gpu.h).
This module is a thin Python mirror of that ABI for tests and benchmarks; the
reference's own host interface (MatShell MatMult, parameters.txt, ev_ts) is the
C++ layer in laph_eigsys_b200/host.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import (LAYOUT_CONF, LAYOUT_EIGEN, LAYOUT_ROWMAJOR, LINKS_BF16, LINKS_FP32, SMEAR_APE, SMEAR_HYP,
                   SMEAR_NONE, SMEAR_STOUT, WINDOW_FIXED, WINDOW_LANCZOS, WINDOW_MLP, LaphError, check, lib)

__all__ = ["Context", "Solver", "gauge_random", "lime_write_gauge", "lime_read_gauge", "lime_read_gauge_any",
           "lime_info", "parse_parameters", "sourceshape", "sourceshape_avg", "write_sourceshape", "check_trace",
           "fix_phase", "reset_phase", "read_eigenvalues_ascii", "write_gauge_matrices", "read_gauge_matrices",
           "recover_spectrum", "write_eigsys_bin", "write_eigenvalues_bin", "read_eigsys_bin",
           "read_eigenvalues_bin", "autotune", "autotune_search", "solver_footprint",
           "solver_max_batch", "LaphError", "lib"]


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def _c128(a):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a


def gauge_random(L, nt, eps, seed):
    """Seeded U = exp(i eps H) links; array (nt, L^3, 4, 3, 3) complex128, slot 0 = U_t."""
    conf = np.empty((nt, L ** 3, 4, 3, 3), dtype=np.complex128)
    check(lib.laph_gauge_random(_ptr(conf), L, nt, eps, seed), "laph_gauge_random")
    return conf


def lime_write_gauge(path, conf, L, T, precision=64):
    """ILDG/LIME file of conf (T, L^3, 4, 3, 3) complex128 (laph_lime_write_gauge_prec), FP64 or FP32 payload."""
    conf = _c128(conf)
    check(lib.laph_lime_write_gauge_prec(str(path).encode(), _ptr(conf), L, T, precision),
          "laph_lime_write_gauge_prec")


def lime_read_gauge(path, T, L, t_i, t_f):
    """Timeslices t_i..t_f of an FP64 ILDG file (read_lime_gauge_field_doubleprec_timeslices, modules/io.cpp:22-146)."""
    conf = np.empty((t_f - t_i + 1, L ** 3, 4, 3, 3), dtype=np.complex128)
    check(lib.laph_lime_read_gauge(str(path).encode(), T, L, t_i, t_f, _ptr(conf)), "laph_lime_read_gauge")
    return conf


def lime_read_gauge_any(path, T, L, t_i, t_f):
    """FP64 or FP32 ILDG links (FP32 widened); returns (conf, precision)."""
    conf = np.empty((t_f - t_i + 1, L ** 3, 4, 3, 3), dtype=np.complex128)
    prec = ctypes.c_int()
    check(lib.laph_lime_read_gauge_any(str(path).encode(), T, L, t_i, t_f, _ptr(conf), ctypes.byref(prec)),
          "laph_lime_read_gauge_any")
    return conf, prec.value


def lime_info(path):
    """(lx, ly, lz, lt, precision) from the ildg-format record."""
    v = [ctypes.c_int() for _ in range(5)]
    check(lib.laph_lime_info(str(path).encode(), *[ctypes.byref(x) for x in v]), "laph_lime_info")
    return tuple(x.value for x in v)


def sourceshape(V, L, evals=None, device=0):
    """psi(r) of an eigensystem V [3 V3][nev] on the grid r_i = 0, 2, ... < L (device kernel)."""
    V = np.asfortranarray(V, dtype=np.complex128)
    psi = np.empty((L // 2) ** 3)
    ev = None if evals is None else np.ascontiguousarray(evals, dtype=np.float64)
    check(lib.laph_sourceshape(ctypes.c_void_p(V.ctypes.data), L, V.shape[1],
                               None if ev is None else _ptr(ev), 0, _ptr(psi), device), "laph_sourceshape")
    return psi


def sourceshape_avg(L, psi):
    """avg_radii: (radii, averaged psi) in order of first appearance."""
    psi = np.ascontiguousarray(psi, dtype=np.float64)
    r = np.empty(len(psi))
    a = np.empty(len(psi))
    n = ctypes.c_int()
    check(lib.laph_sourceshape_avg(L, _ptr(psi), _ptr(r), _ptr(a), ctypes.byref(n)), "laph_sourceshape_avg")
    return r[:n.value], a[:n.value]


def write_sourceshape(dirname, config, t, nev, r, psi):
    """write_sourceshape_ascii / _bin (modules/read_write.cpp:205-234): the radius-averaged psi(r) files."""
    r = np.ascontiguousarray(r, dtype=np.float64)
    psi = np.ascontiguousarray(psi, dtype=np.float64)
    check(lib.laph_write_sourceshape(str(dirname).encode() if dirname else None, config, t, nev, len(r), _ptr(r),
                                     _ptr(psi)), "laph_write_sourceshape")


def spatial_links(conf_ts):
    """(V3, 4, 3, 3) conf timeslice -> (V3, 3, 3, 3) spatial links (map_timeslice_to_eigen)."""
    return np.ascontiguousarray(np.asarray(conf_ts)[:, 1:4])


def timeslice_split(LT, size, rank):
    """(t0, count) of rank's contiguous timeslice block (the reference's MPI split)."""
    t0, n = ctypes.c_int(), ctypes.c_int()
    check(lib.laph_timeslice_split(LT, size, rank, ctypes.byref(t0), ctypes.byref(n)), "laph_timeslice_split")
    return t0.value, n.value


def parse_parameters(path):
    """parameters.txt as IO::set_values reads it (modules/par_io.cpp:8-136), plus this library's keys; a dict."""
    cfg = _lib.laph_config()
    check(lib.laph_parse_parameters(str(path).encode(), ctypes.byref(cfg)), "laph_parse_parameters")
    out = {}
    for name, _ in cfg._fields_:
        v = getattr(cfg, name)
        out[name] = v.decode() if isinstance(v, bytes) else v
    return out


def check_trace(V):
    """check_trace (modules/read_write.cpp:20-35): (passes, tr(V^dag V), sum(V^dag V))."""
    V = np.asfortranarray(V, dtype=np.complex128)
    dim, nev = V.shape
    tr, sm = ctypes.c_double(), ctypes.c_double()
    ok = lib.laph_check_trace(dim, nev, ctypes.c_void_p(V.ctypes.data), ctypes.byref(tr), ctypes.byref(sm))
    return bool(ok), tr.value, sm.value


def fix_phase(V):
    """fix_phase (modules/eigensystem.cpp:4-30): (V with every first entry real >= 0, the removed phases)."""
    V = np.asfortranarray(V, dtype=np.complex128)
    dim, nev = V.shape
    Vf = np.empty_like(V, order="F")
    ph = np.empty(nev)
    check(lib.laph_fix_phase_host(dim, nev, ctypes.c_void_p(V.ctypes.data), ctypes.c_void_p(Vf.ctypes.data),
                                  _ptr(ph)), "laph_fix_phase_host")
    return Vf, ph


def reset_phase(V, phase_want):
    """reset_phase: column n rotated so that its first entry has phase phase_want[n]."""
    V = np.asfortranarray(V, dtype=np.complex128)
    dim, nev = V.shape
    want = np.ascontiguousarray(phase_want, dtype=np.float64)
    Vr = np.empty_like(V, order="F")
    check(lib.laph_reset_phase_host(dim, nev, ctypes.c_void_p(V.ctypes.data), _ptr(want),
                                    ctypes.c_void_p(Vr.ctypes.data)), "laph_reset_phase_host")
    return Vr


def read_eigenvalues_ascii(prefix, config, t, nev):
    """read_eigenvalues_ascii: nev values from "<prefix>.%03d.%04d" (timeslice, configuration)."""
    ev = np.empty(nev)
    check(lib.laph_read_eigenvalues_ascii(str(prefix).encode(), config, t, nev, _ptr(ev)),
          "laph_read_eigenvalues_ascii")
    return ev


def write_gauge_matrices(path, G):
    """write_gauge_matrices: (V3, 3, 3) complex128 matrices as raw Eigen (column-major) Matrix3cd."""
    G = np.asarray(G, dtype=np.complex128)
    raw = np.ascontiguousarray(np.swapaxes(G, 1, 2))  # row-major (a, b) -> column-major memory
    check(lib.laph_write_gauge_matrices(str(path).encode(), G.shape[0], _ptr(raw)), "laph_write_gauge_matrices")


def read_gauge_matrices(path, V3):
    """read_gauge_matrices: (V3, 3, 3) complex128 matrices from raw Eigen (column-major) Matrix3cd."""
    raw = np.empty((V3, 3, 3), dtype=np.complex128)
    check(lib.laph_read_gauge_matrices(str(path).encode(), V3, _ptr(raw)), "laph_read_gauge_matrices")
    return np.ascontiguousarray(np.swapaxes(raw, 1, 2))


def recover_spectrum(theta, deg, lam_l, lam_c):
    """recover_spectrum (modules/recover_spec.cpp:13-54): stored eigenvalues (of Delta, <= 0) from T_deg(B) ones."""
    theta = np.ascontiguousarray(theta, dtype=np.float64)
    out = np.empty_like(theta)
    check(lib.laph_recover_spectrum(len(theta), _ptr(theta), deg, lam_l, lam_c, _ptr(out)), "laph_recover_spectrum")
    return out


def write_eigsys_bin(dirname, prefix, config, t, V):
    """write_eig_sys_bin (modules/read_write.cpp:176-201): "<dir>/<prefix>.%04d.%03d", check_trace first."""
    V = np.asfortranarray(V, dtype=np.complex128)
    check(lib.laph_write_eigsys_bin(str(dirname).encode(), prefix.encode(), config, t, V.shape[0], V.shape[1],
                                    ctypes.c_void_p(V.ctypes.data)), "laph_write_eigsys_bin")


def write_eigenvalues_bin(dirname, prefix, config, t, ev):
    """write_eigenvalues_bin (modules/read_write.cpp:237-250): raw doubles to "<dir>/<prefix>.%04d.%03d"."""
    ev = np.ascontiguousarray(ev, dtype=np.float64)
    check(lib.laph_write_eigenvalues_bin(str(dirname).encode(), prefix.encode(), config, t, len(ev), _ptr(ev)),
          "laph_write_eigenvalues_bin")


def read_eigsys_bin(dirname, prefix, config, t, dim, nev):
    """read_evectors_bin_ts (modules/read_write.cpp:70-97): [dim][nev] column-major block, check_trace applied."""
    V = np.empty((dim, nev), dtype=np.complex128, order="F")
    check(lib.laph_read_eigsys_bin(str(dirname).encode(), prefix.encode(), config, t, dim, nev,
                                   ctypes.c_void_p(V.ctypes.data)), "laph_read_eigsys_bin")
    return V


def read_eigenvalues_bin(dirname, prefix, config, t, nev):
    """read_eigenvalues_bin (modules/read_write.cpp:135-152): nev raw doubles."""
    ev = np.empty(nev)
    check(lib.laph_read_eigenvalues_bin(str(dirname).encode(), prefix.encode(), config, t, nev, _ptr(ev)),
          "laph_read_eigenvalues_bin")
    return ev


class Context:
    """One timeslice on one device: the MatShell drop-in (laph_ctx)."""

    def __init__(self, L, lam_l=11.8, lam_c=0.6, deg=8, device=0):
        self.L, self.V3, self.dim = L, L ** 3, 3 * L ** 3
        p = _lib.laph_params(L, lam_l, lam_c, deg, device)
        h = ctypes.c_void_p()
        check(lib.laph_ctx_create(ctypes.byref(h), ctypes.byref(p)), "laph_ctx_create")
        self._h = h
        self.deg = deg

    def close(self):
        """Free the context's device memory and stream (laph_ctx_destroy)."""
        if self._h:
            lib.laph_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_window(self, lam_l, lam_c, deg):
        """LAM_L, LAM_C and DEG of the MatShell product (laph_ctx_set_window)."""
        check(lib.laph_ctx_set_window(self._h, lam_l, lam_c, deg), "laph_ctx_set_window")
        self.deg = deg

    def set_links(self, links, layout=LAYOUT_ROWMAJOR):
        """Host links of the timeslice (laph_set_links; map_timeslice_to_eigen for LAYOUT_CONF)."""
        links = _c128(links)
        check(lib.laph_set_links(self._h, _ptr(links), layout), "laph_set_links")

    def get_links(self, layout=LAYOUT_ROWMAJOR):
        """The (smeared) links back on the host (laph_get_links; Tslice::get_gauge)."""
        shape = (self.V3, 4, 3, 3) if layout == LAYOUT_CONF else (self.V3, 3, 3, 3)
        out = np.empty(shape, dtype=np.complex128)
        check(lib.laph_get_links(self._h, _ptr(out), layout), "laph_get_links")
        return out

    def smear(self, kind, p1, p2, iters, compat=1):
        """FP64 smearing on the device (laph_smear): kind SMEAR_HYP / SMEAR_STOUT / SMEAR_APE."""
        check(lib.laph_smear(self._h, kind, p1, p2, iters, compat), "laph_smear")

    def smearing_hyp(self, alpha_1, alpha_2, iters):
        """Tslice::smearing_hyp (modules/timeslice.cpp:243-369) on the device."""
        self.smear(SMEAR_HYP, alpha_1, alpha_2, iters, 0)

    def smearing_stout(self, rho, iters, compat=1):
        """Tslice::smearing_stout (modules/timeslice.cpp:145-193); compat keeps its backward-staple factor."""
        self.smear(SMEAR_STOUT, rho, 0.0, iters, compat)

    def smearing_ape(self, alpha, iters, compat=1):
        """Tslice::smearing_ape (modules/timeslice.cpp:196-239); compat keeps its backward-staple factor."""
        self.smear(SMEAR_APE, alpha, 0.0, iters, compat)

    def matmult(self, x, deg=None):
        """y = T_deg(B) x in FP64, the MatShell product (MatMult_Laplacian2D / tv_iter), host vectors."""
        x = _c128(x)
        y = np.empty_like(x)
        check(lib.laph_matmult(self._h, _ptr(x), _ptr(y), self.deg if deg is None else deg, 0), "laph_matmult")
        return y

    def stream(self):
        """The context's CUDA stream handle (laph_ctx_stream), for timing its products with events."""
        h = ctypes.c_void_p()
        check(lib.laph_ctx_stream(self._h, ctypes.byref(h)), "laph_ctx_stream")
        return h.value or 0

    def matmult_device(self, x_ptr, y_ptr, deg=None):
        """As matmult on device pointers (complex128[3 V3] each)."""
        check(lib.laph_matmult(self._h, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr),
                               self.deg if deg is None else deg, 1), "laph_matmult")

    def apply_neglap(self, x):
        """(-Delta) x = 6 x - hop(x) in FP64 (laph_apply_neglap)."""
        x = _c128(x)
        y = np.empty_like(x)
        check(lib.laph_apply_neglap(self._h, _ptr(x), _ptr(y), 0), "laph_apply_neglap")
        return y

    def get_diagonal(self):
        """MatGetDiagonal_Laplacian2D (modules/shell_matop.cpp:248-255): the constant -6."""
        d = np.empty(self.dim, dtype=np.complex128)
        check(lib.laph_get_diagonal(self._h, _ptr(d), 0), "laph_get_diagonal")
        return d

    def eps_solve(self, nev, ncv=0, tol=1e-10, max_it=100, device_basis=True, seed=1227, vectors=True):
        """Plain form: Krylov-Schur on T_deg(B) driving this context's MatMult (laph_eps_solve).
        Returns (status, theta[nev], V or None, nconv, restarts, nmatvec)."""
        theta = np.empty(nev)
        V = np.empty((self.dim, nev), dtype=np.complex128, order="F") if vectors else None
        nconv, its, nmv = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
        st = lib.laph_eps_solve(self._h, nev, ncv, tol, max_it, int(device_basis), seed, _ptr(theta),
                                ctypes.c_void_p(V.ctypes.data) if vectors else None, ctypes.byref(nconv),
                                ctypes.byref(its), ctypes.byref(nmv))
        if st not in (_lib.LAPH_OK, _lib.LAPH_ENOTCONV):
            check(st, "laph_eps_solve")
        return st, theta, V, nconv.value, its.value, nmv.value

    def displace(self, V, direction):
        """Covariant displacement of the columns of V along direction 0/1/2 with this context's links."""
        V = np.asfortranarray(V, dtype=np.complex128)
        W = np.empty_like(V, order="F")
        check(lib.laph_displace(self._h, direction, ctypes.c_void_p(V.ctypes.data), ctypes.c_void_p(W.ctypes.data),
                                V.shape[1], 0), "laph_displace")
        return W

    def plaquette(self):
        """Average spatial plaquette (plaque_timeslice, modules/config_utils.cpp:388-426)."""
        p = ctypes.c_double()
        check(lib.laph_plaquette(self._h, ctypes.byref(p)), "laph_plaquette")
        return p.value


def _tune_dict(r):
    return {f: getattr(r, f) for f, _ in r._fields_}


def _probs(problems):
    probs = [(int(L), int(n)) for L, n in problems]
    return (_lib.laph_problem * len(probs))(*[_lib.laph_problem(L, n) for L, n in probs]), len(probs)


def solver_footprint(problems, opts=None, **kw):
    """Device bytes laph_solver_create would allocate for these problems."""
    arr, n = _probs(problems)
    o = opts if opts is not None else solve_opts(**kw)
    b = ctypes.c_longlong()
    check(lib.laph_solver_footprint(arr, n, ctypes.byref(o), ctypes.byref(b)), "laph_solver_footprint")
    return b.value


def solver_max_batch(problems, opts=None, device=0, fraction=0.85, **kw):
    """Largest leading count of problems whose solver fits in `fraction` of the device's free memory."""
    arr, n = _probs(problems)
    o = opts if opts is not None else solve_opts(**kw)
    m = ctypes.c_int()
    check(lib.laph_solver_max_batch(arr, n, ctypes.byref(o), device, fraction, ctypes.byref(m)),
          "laph_solver_max_batch")
    return m.value


def autotune_search(deg_c, block_c, guard_c, start, trial):
    """laph_autotune_search with a Python trial(deg, block, guard) -> ms per problem (< 0: failed)."""
    arr = lambda v: (ctypes.c_int * max(len(v), 1))(*v)  # noqa: E731
    cb = _lib.TUNE_TRIAL(lambda user, d, b, g: float(trial(d, b, g)))
    r = _lib.laph_tune_result()
    check(lib.laph_autotune_search(arr(deg_c), len(deg_c), arr(block_c), len(block_c), arr(guard_c), len(guard_c),
                                   start[0], start[1], start[2], cb, None, ctypes.byref(r)), "laph_autotune_search")
    return _tune_dict(r)


def autotune(problems, links, nsample=4, cache=None, device=0, layout=LAYOUT_ROWMAJOR, opts=None, model=None, **kw):
    """laph_solver_autotune: (tuned laph_solve_opts, result dict) for a batch shaped like `problems`, timed on
    the first min(len(problems), nsample) problems with their host links; model: the window model (float32) for
    window = WINDOW_MLP."""
    probs = [(int(L), int(n)) for L, n in problems]
    arr = (_lib.laph_problem * len(probs))(*[_lib.laph_problem(L, n) for L, n in probs])
    o = opts if opts is not None else solve_opts(**kw)
    ns = min(len(probs), nsample)
    keep = [_c128(links[i]) for i in range(ns)]
    ptrs = (ctypes.c_void_p * ns)(*[ctypes.c_void_p(a.ctypes.data) for a in keep])
    m = None if model is None else np.ascontiguousarray(model, dtype=np.float32)
    r = _lib.laph_tune_result()
    check(lib.laph_solver_autotune(arr, len(probs), ptrs, layout, nsample, ctypes.byref(o),
                                   None if m is None else ctypes.c_void_p(m.ctypes.data), 0 if m is None else m.size,
                                   device, str(cache).encode() if cache else None, ctypes.byref(r)),
          "laph_solver_autotune")
    return o, _tune_dict(r)


def probe_fp64(device=0):
    """(FP64 FMA TFLOP/s, FP64 tensor-path DMMA TFLOP/s) measured in place on the device (laph_probe_fp64)."""
    a, b = ctypes.c_double(), ctypes.c_double()
    check(lib.laph_probe_fp64(device, ctypes.byref(a), ctypes.byref(b)), "laph_probe_fp64")
    return a.value, b.value


def check_report(reset=False):
    """Indices found out of range by the bounds-checked build (laph_check_report): a dict with the count and, when
    it is not zero, the first one's value, bound, source line and translation unit.  Always a count of 0 in the
    normal build (check_enabled() tells which build is loaded)."""
    n, i, b, ln = ctypes.c_uint64(), ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_int()
    unit = ctypes.create_string_buffer(256)
    check(lib.laph_check_report(ctypes.byref(n), ctypes.byref(i), ctypes.byref(b), ctypes.byref(ln), unit, 256,
                                1 if reset else 0), "laph_check_report")
    out = {"count": n.value}
    if n.value:
        out.update(index=i.value, bound=b.value, line=ln.value, unit=unit.value.decode())
    return out


def check_enabled():
    """True when the loaded library is the bounds-checked build (LAPH_GPU_LIB=check)."""
    return bool(lib.laph_check_enabled())


def solve_opts(**kw):
    o = _lib.laph_solve_opts()
    lib.laph_solve_opts_default(ctypes.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


class Solver:
    """Batched block eigensolver over many timeslices (laph_solver)."""

    def __init__(self, problems, opts=None, device=0, **kw):
        self.problems = [(int(L), int(nev)) for L, nev in problems]
        arr = (_lib.laph_problem * len(self.problems))(*[_lib.laph_problem(L, n) for L, n in self.problems])
        self.opts = opts if opts is not None else solve_opts(**kw)
        h = ctypes.c_void_p()
        check(lib.laph_solver_create(ctypes.byref(h), arr, len(self.problems), ctypes.byref(self.opts), device),
              "laph_solver_create")
        self._h = h

    def close(self):
        """Free the solver's device memory, graphs and stream (laph_solver_destroy)."""
        if self._h:
            lib.laph_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_links(self, i, links, layout=LAYOUT_ROWMAJOR):
        """Host links of problem i (laph_solver_set_links); non-finite entries are refused."""
        links = _c128(links)
        check(lib.laph_solver_set_links(self._h, i, _ptr(links), layout, 0), "laph_solver_set_links")

    def set_links_device(self, i, ptr, layout=LAYOUT_ROWMAJOR):
        """Links of problem i from device memory at ptr (ROWMAJOR or CONF)."""
        check(lib.laph_solver_set_links(self._h, i, ctypes.c_void_p(ptr), layout, 1), "laph_solver_set_links")

    def run(self):
        """(status, per-problem result dicts) of one smear + solve of every problem (laph_solver_run)."""
        res = (_lib.laph_result * len(self.problems))()
        st = lib.laph_solver_run(self._h, res)
        if st not in (_lib.LAPH_OK, _lib.LAPH_ENOTCONV):
            check(st, "laph_solver_run")
        return st, [dict((f, getattr(r, f)) for f, _ in r._fields_) for r in res]

    def get(self, i, vectors=True):
        """(eigenvalues as the reference stores them, phase-fixed eigenvectors [3 V3][nev] or None, phases) of
        problem i."""
        L, nev = self.problems[i]
        ev = np.empty(nev)
        V = np.empty((3 * L ** 3, nev), dtype=np.complex128, order="F") if vectors else None
        ph = np.empty(nev)
        check(lib.laph_solver_get(self._h, i, _ptr(ev), ctypes.c_void_p(V.ctypes.data) if vectors else None,
                                  _ptr(ph), 0), "laph_solver_get")
        return ev, V, ph

    def stream(self):
        """The solver's CUDA stream handle (an int), for timing or ordering work around run()."""
        h = ctypes.c_void_p()
        check(lib.laph_solver_stream(self._h, ctypes.byref(h)), "laph_solver_stream")
        return h.value

    def get_into(self, i, evals, evecs, phases):
        """Fetch problem i into caller-provided host arrays (e.g. pinned)."""
        check(lib.laph_solver_get(self._h, i, _ptr(evals), ctypes.c_void_p(evecs.ctypes.data) if evecs is not None
                                  else None, _ptr(phases), 0), "laph_solver_get")

    def get_async(self, i, evals, evecs, phases):
        """Queue problem i's results into caller-provided host arrays (pinned for overlap) on the solver's read-back
        stream (laph_solver_get_async); they are complete after wait()."""
        check(lib.laph_solver_get_async(self._h, i, _ptr(evals) if evals is not None else None,
                                        ctypes.c_void_p(evecs.ctypes.data) if evecs is not None else None,
                                        _ptr(phases) if phases is not None else None), "laph_solver_get_async")

    def ritz(self, i):
        """All k Ritz values of problem i's block after the last run (the nev wanted ones and the guard), ascending
        (laph_solver_ritz)."""
        th = np.empty(512)
        k = ctypes.c_int()
        check(lib.laph_solver_ritz(self._h, i, _ptr(th), ctypes.byref(k)), "laph_solver_ritz")
        return np.sort(th[:k.value])

    def wait(self):
        """Block until every queued read-back has landed (laph_solver_wait)."""
        check(lib.laph_solver_wait(self._h), "laph_solver_wait")

    def timings(self):
        """Device ms of the last run: smearing + setup, filter, dense + FP64 stencils, total."""
        t = (ctypes.c_double * 4)()
        check(lib.laph_solver_timings(self._h, t), "laph_solver_timings")
        return list(t)

    def displace(self, i, direction):
        """Covariant displacement of problem i's eigenvectors along direction 0/1/2 (device, FP64)."""
        L, nev = self.problems[i]
        W = np.empty((3 * L ** 3, nev), dtype=np.complex128, order="F")
        check(lib.laph_solver_displace(self._h, i, direction, ctypes.c_void_p(W.ctypes.data), 0),
              "laph_solver_displace")
        return W

    def displace_device(self, i, direction, ptr):
        """As displace(), writing [3 V3][nev] complex128 to device memory at ptr."""
        check(lib.laph_solver_displace(self._h, i, direction, ctypes.c_void_p(ptr), 1), "laph_solver_displace")

    def set_smear(self, i, p1, p2=0.0):
        """Smearing parameters of problem i only (the batched tune_hyp scan)."""
        check(lib.laph_solver_set_smear(self._h, i, p1, p2), "laph_solver_set_smear")

    def sourceshape(self, i, weighted=False):
        """psi(r) of problem i's eigenvectors, computed on the device from the solver's own block."""
        L = self.problems[i][0]
        psi = np.empty((L // 2) ** 3)
        check(lib.laph_solver_sourceshape(self._h, i, int(bool(weighted)), _ptr(psi)), "laph_solver_sourceshape")
        return psi

    def counters(self):
        """Filter site-vector-steps, filter launches and all kernel launches of the last run."""
        c = (ctypes.c_longlong * 3)()
        check(lib.laph_solver_counters(self._h, c), "laph_solver_counters")
        return list(c)

    def loop_info(self):
        """(device_loop, graph launches) of the last run (laph_solver_loop_info)."""
        a, b = ctypes.c_int(), ctypes.c_longlong()
        check(lib.laph_solver_loop_info(self._h, ctypes.byref(a), ctypes.byref(b)), "laph_solver_loop_info")
        return a.value, b.value

    def filter_bytes(self):
        """Algorithmic bytes of the last run's filter passes (laph_solver_filter_bytes): (correction form as
        run, 72 B + links per site-vector-step)."""
        c = (ctypes.c_double * 2)()
        check(lib.laph_solver_filter_bytes(self._h, c), "laph_solver_filter_bytes")
        return list(c)
