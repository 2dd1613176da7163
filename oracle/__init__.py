"""ctypes wrapper of the CPU FP64 oracle (oracle/liblaph_oracle.so).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the CPU
baseline leg of bench.py as the checker / timed CPU baseline, never by the
product path.  Parity status: arithmetic unpinned against reference outputs
(the reference cannot be built here as a whole and ships no golden vectors);
site indexing and formulas checked on the reference's compiled parameter parser
and lookup tables (oracle/_ref/ref_dump), and pinned by analytic known answers
(see laph_oracle.h).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblaph_oracle.so")


def build():
    subprocess.run(["make", "-C", _HERE], check=True, stdout=subprocess.DEVNULL)


if not os.path.exists(LIB_PATH):
    build()

_lib = ctypes.CDLL(LIB_PATH)
_d, _i, _vp = ctypes.c_double, ctypes.c_int, ctypes.c_void_p


def _sig(name, res, *args):
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = list(args)


_sig("orc_set_threads", None, _i)
_sig("orc_lime_read_gauge", _i, ctypes.c_char_p, _i, _i, _i, _i, _vp)
_sig("orc_map_timeslice", None, _vp, _i, _vp)
_sig("orc_proj_su3", None, _vp)
_sig("orc_expiH", None, _vp, _vp)
_sig("orc_gauge_random", None, _vp, _i, _i, _d, ctypes.c_uint64)
_sig("orc_smear_stout", None, _vp, _i, _d, _i, _i)
_sig("orc_smear_ape", None, _vp, _i, _d, _i, _i)
_sig("orc_smear_hyp", None, _vp, _i, _d, _d, _i)
_sig("orc_tv2", None, _vp, _i, _d, _d, _vp, _vp)
_sig("orc_tv_iter", None, _vp, _i, _d, _d, _i, _vp, _vp)
_sig("orc_neglap", None, _vp, _i, _vp, _vp)
_sig("orc_plaquette", _d, _vp, _i)
_sig("orc_eps_solve", _i, _vp, _i, _d, _d, _i, _i, _i, _d, _i, ctypes.c_uint64, _vp, _vp,
     ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(ctypes.c_longlong))
_sig("orc_recover_spectrum", None, _i, _vp, _i, _d, _d, _vp)
_sig("orc_fix_phase", None, _i, _i, _vp, _vp, _vp)
_sig("orc_reset_phase", None, _i, _i, _vp, _vp, _vp)
_sig("orc_build_neglap_dense", None, _vp, _i, _vp)
_sig("orc_mlp_loss_grad", _d, _vp, _vp, _vp, _i, _vp)
_sig("orc_sourceshape", None, _vp, _i, _i, _vp)
_sig("orc_displace", None, _vp, _i, _i, _vp, _i, _vp)
_sig("orc_sourceshape_avg", _i, _i, _vp, _vp, _vp)


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def _links(U):
    return np.ascontiguousarray(U, dtype=np.complex128).copy()


def set_threads(n):
    _lib.orc_set_threads(int(n))


def lime_read_gauge(path, T, L, t_i, t_f):
    conf = np.zeros((t_f - t_i + 1, L ** 3, 4, 3, 3), dtype=np.complex128)
    st = _lib.orc_lime_read_gauge(str(path).encode(), T, L, t_i, t_f, _p(conf))
    return st, conf


def map_timeslice(conf_ts, L):
    conf_ts = np.ascontiguousarray(conf_ts, dtype=np.complex128)
    out = np.empty((L ** 3, 3, 3, 3), dtype=np.complex128)
    _lib.orc_map_timeslice(_p(conf_ts), L, _p(out))
    return out


def proj_su3(m):
    m = np.ascontiguousarray(m, dtype=np.complex128).copy()
    _lib.orc_proj_su3(_p(m))
    return m


def expiH(h):
    h = np.ascontiguousarray(h, dtype=np.complex128)
    out = np.empty((3, 3), dtype=np.complex128)
    _lib.orc_expiH(_p(h), _p(out))
    return out


def gauge_random(L, nt, eps, seed):
    """Seeded synthetic gauge field (nt, V3, 4, 3, 3) complex128, U = exp(i eps H) (orc_gauge_random)."""
    conf = np.empty((nt, L ** 3, 4, 3, 3), dtype=np.complex128)
    _lib.orc_gauge_random(_p(conf), L, nt, eps, seed)
    return conf


def smear_stout(U, L, rho, iters, compat=1):
    U = _links(U)
    _lib.orc_smear_stout(_p(U), L, rho, iters, compat)
    return U


def smear_ape(U, L, alpha, iters, compat=1):
    U = _links(U)
    _lib.orc_smear_ape(_p(U), L, alpha, iters, compat)
    return U


def smear_hyp(U, L, a1, a2, iters):
    U = _links(U)
    _lib.orc_smear_hyp(_p(U), L, a1, a2, iters)
    return U


def tv2(U, L, lam_l, lam_c, x):
    U = np.ascontiguousarray(U, dtype=np.complex128)
    x = np.ascontiguousarray(x, dtype=np.complex128)
    y = np.zeros_like(x)
    _lib.orc_tv2(_p(U), L, lam_l, lam_c, _p(x), _p(y))
    return y


def tv_iter(U, L, lam_l, lam_c, deg, x, y=None):
    U = np.ascontiguousarray(U, dtype=np.complex128)
    x = np.ascontiguousarray(x, dtype=np.complex128)
    y = np.zeros_like(x) if y is None else np.ascontiguousarray(y, dtype=np.complex128).copy()
    _lib.orc_tv_iter(_p(U), L, lam_l, lam_c, deg, _p(x), _p(y))
    return y


def neglap(U, L, x):
    U = np.ascontiguousarray(U, dtype=np.complex128)
    x = np.ascontiguousarray(x, dtype=np.complex128)
    y = np.zeros_like(x)
    _lib.orc_neglap(_p(U), L, _p(x), _p(y))
    return y


def plaquette(U, L):
    U = np.ascontiguousarray(U, dtype=np.complex128)
    return _lib.orc_plaquette(_p(U), L)


def eps_solve(U, L, lam_l, lam_c, deg, nev, ncv=0, tol=1e-12, max_it=200, seed=1227):
    """SLEPc-style Krylov-Schur on T_deg(B), largest magnitude.  Returns
    (status, theta[nev], V (dim x nev, column-major), nconv, its, nmatvec)."""
    U = np.ascontiguousarray(U, dtype=np.complex128)
    dim = 3 * L ** 3
    theta = np.zeros(nev)
    V = np.zeros((dim, nev), dtype=np.complex128, order="F")
    nconv, its, nmv = _i(), _i(), ctypes.c_longlong()
    st = _lib.orc_eps_solve(_p(U), L, lam_l, lam_c, deg, nev, ncv, tol, max_it, seed, _p(theta),
                            ctypes.c_void_p(V.ctypes.data), ctypes.byref(nconv), ctypes.byref(its), ctypes.byref(nmv))
    return st, theta, V, nconv.value, its.value, nmv.value


def recover_spectrum(theta, deg, lam_l, lam_c):
    theta = np.ascontiguousarray(theta, dtype=np.float64)
    out = np.empty_like(theta)
    _lib.orc_recover_spectrum(len(theta), _p(theta), deg, lam_l, lam_c, _p(out))
    return out


def fix_phase(V):
    V = np.asfortranarray(V, dtype=np.complex128)
    dim, nev = V.shape
    Vf = np.empty_like(V, order="F")
    ph = np.empty(nev)
    _lib.orc_fix_phase(dim, nev, ctypes.c_void_p(V.ctypes.data), ctypes.c_void_p(Vf.ctypes.data), _p(ph))
    return Vf, ph


def reset_phase(V, phase_want):
    V = np.asfortranarray(V, dtype=np.complex128)
    dim, nev = V.shape
    want = np.ascontiguousarray(phase_want, dtype=np.float64)
    Vr = np.empty_like(V, order="F")
    _lib.orc_reset_phase(dim, nev, ctypes.c_void_p(V.ctypes.data), _p(want), ctypes.c_void_p(Vr.ctypes.data))
    return Vr


def neglap_dense(U, L):
    U = np.ascontiguousarray(U, dtype=np.complex128)
    dim = 3 * L ** 3
    A = np.zeros((dim, dim), dtype=np.complex128)
    _lib.orc_build_neglap_dense(_p(U), L, _p(A))
    return A


def displace(U, L, direction, V):
    """right_displacement_one_dir: W = (U V(x+dir) - U(x-dir)^dag V(x-dir)) / 2 for every column."""
    U = np.ascontiguousarray(U, dtype=np.complex128)
    V = np.asfortranarray(V, dtype=np.complex128)
    W = np.empty_like(V, order="F")
    _lib.orc_displace(_p(U), L, direction, ctypes.c_void_p(V.ctypes.data), V.shape[1], ctypes.c_void_p(W.ctypes.data))
    return W


def sourceshape(V, L):
    """psi(r) on the grid r_i = 0, 2, ... < L (r1 outer, r3 inner)."""
    V = np.asfortranarray(V, dtype=np.complex128)
    n = ((L + 1) // 2) ** 3
    psi = np.empty(n)
    _lib.orc_sourceshape(ctypes.c_void_p(V.ctypes.data), L, V.shape[1], _p(psi))
    return psi


def sourceshape_avg(L, psi):
    """avg_radii: (radii, psi averages) in order of first appearance."""
    psi = np.ascontiguousarray(psi, dtype=np.float64)
    r = np.empty(len(psi))
    a = np.empty(len(psi))
    n = _lib.orc_sourceshape_avg(L, _p(psi), _p(r), _p(a))
    return r[:n], a[:n]


def free_spectrum(L):
    """Analytic spectrum of -Delta for U = 1: sum_i 4 sin^2(pi n_i / L), x3 colours."""
    k = 4.0 * np.sin(np.pi * np.arange(L) / L) ** 2
    ev = (k[:, None, None] + k[None, :, None] + k[None, None, :]).ravel()
    return np.sort(np.repeat(ev, 3))


def mlp_loss_grad(params, X, Y):
    """FP64 loss and gradient of the window MLP (16->64->64->3, tanh)."""
    P = np.ascontiguousarray(params, dtype=np.float64)
    X = np.ascontiguousarray(X, dtype=np.float64)
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    g = np.zeros_like(P)
    loss = _lib.orc_mlp_loss_grad(_p(P), _p(X), _p(Y), X.shape[0], _p(g))
    return loss, g


def rayleigh(U, L, V):
    """FP64 Rayleigh quotients lambda_j = v_j^H (-Delta) v_j / v_j^H v_j of the columns of V on links U, and their
    residual norms ||(-Delta) v_j - lambda_j v_j|| / ||v_j|| (the oracle's stencil)."""
    V = np.asarray(V)
    lam = np.empty(V.shape[1])
    res = np.empty(V.shape[1])
    for j in range(V.shape[1]):
        v = np.ascontiguousarray(V[:, j])
        y = neglap(U, L, v)
        n2 = np.vdot(v, v).real
        lam[j] = np.vdot(v, y).real / n2
        res[j] = np.linalg.norm(y - lam[j] * v) / np.sqrt(n2)
    return lam, res


def _subspace_distance(A, B):
    """sin of the largest principal angle between span(A) and span(B) (orthonormal columns): ||A - B (B^H A)||_2."""
    return float(np.linalg.norm(A - B @ (B.conj().T @ A), 2))


def compare_eigensystems(U, L, Va, Vb, lam_max=12.0, gap=1e-3, lam_next=None):
    """Eigenpair parity of two eigensystems Va (the one checked) and Vb (the oracle's) of -Delta on links U, both
    (dim, nev) column-major with the reference's phase fix applied (fix_phase).  Eigenvalues are compared as FP64
    Rayleigh quotients on -Delta, each relative to itself (where lambda > 1e-12 lambda_max) and relative to
    lambda_max; eigenvectors one by one where the eigenvalue is isolated (no neighbour within `gap`, absolute, in
    units of lambda), and by subspace distance (sin of the largest principal angle) on clusters of eigenvalues
    closer than `gap`.  `gap_min` is the smallest separation of an isolated eigenvalue: an eigenvector with residual
    r is determined to about r / gap_min, which bounds what any two solvers can agree to.  lam_next: the next
    eigenvalue beyond the block, where known; a last cluster that it joins is cut by the block boundary, so the two
    blocks may hold different vectors of it, and it is left out of the vector comparison (boundary_cut)."""
    la, ra = rayleigh(U, L, Va)
    lb, rb = rayleigh(U, L, Vb)
    ia, ib = np.argsort(la), np.argsort(lb)
    la, ra, lb, rb = la[ia], ra[ia], lb[ib], rb[ib]
    Va, Vb = np.asarray(Va)[:, ia], np.asarray(Vb)[:, ib]
    pos = lb > 1e-12 * lam_max
    out = {"nev": int(len(lb)),
           "max_rel_eig": float(np.max(np.abs(la - lb)[pos] / lb[pos])) if pos.any() else 0.0,
           "max_eig_over_lam_max": float(np.max(np.abs(la - lb)) / lam_max),
           "max_resid_checked": float(ra.max() / lam_max), "max_resid_oracle": float(rb.max() / lam_max),
           "trace_vdv_checked": float(np.sum(np.abs(Va) ** 2)), "trace_vdv_oracle": float(np.sum(np.abs(Vb) ** 2))}
    # clusters on the oracle's eigenvalues
    cl, cur = [], [0]
    for j in range(1, len(lb)):
        if lb[j] - lb[j - 1] < gap:
            cur.append(j)
        else:
            cl.append(cur)
            cur = [j]
    cl.append(cur)
    vec, vec_al, proj, gmin = 0.0, 0.0, 0.0, np.inf
    cut = lam_next is not None and lam_next - lb[-1] < gap
    if cut:
        cl = cl[:-1]
    for c in cl:
        if len(c) == 1:
            j = c[0]
            g = lb[j] - lb[j - 1] if j > 0 else np.inf
            if j + 1 < len(lb):
                g = min(g, lb[j + 1] - lb[j])
            elif lam_next is not None:
                g = min(g, lam_next - lb[j])
            gmin = min(gmin, g)
            a, b = Va[:, j], Vb[:, j]
            vec = max(vec, float(np.linalg.norm(a - b)))
            ph = np.vdot(a, b)
            vec_al = max(vec_al, float(np.linalg.norm(a * (ph / abs(ph)) - b)))
        else:
            proj = max(proj, _subspace_distance(Va[:, c], Vb[:, c]))
    out.update({"clusters": int(sum(len(c) > 1 for c in cl)), "in_clusters": int(sum(len(c) for c in cl if len(c) > 1)),
                "max_vec_phase_fixed": vec, "max_vec_aligned": vec_al, "max_cluster_proj": proj,
                "gap_min_isolated": float(gmin) if np.isfinite(gmin) else None,
                "block_proj": _subspace_distance(Va, Vb), "cluster_gap": gap, "boundary_cut": bool(cut)})
    return out
