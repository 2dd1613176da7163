"""Compare two eigensystem directories timeslice by timeslice: the check a user
runs when switching from LapH_EigSys, with one set of files written by it and
one by laph_ev_ts.  It prints what the reference's test_eigensystems printed
(src/test_eigensystems.cpp: tr and sum of U^dag V, sum |U^dag V|^2, and the
same for U^dag U and V^dag V) and adds the numbers that decide parity:

  dlam      max |lambda_U - lambda_V| / 12 over the nev eigenvalues
  proj      ||U U^dag - V V^dag||_2 over the eigenvalue clusters that the nev
            columns contain completely (gap < 1e-6 * 12 inside a cluster), from
            the principal angles between the two subspaces
  phase     max |arg U(0, n)| and |arg V(0, n)|: 0 for phase-fixed vectors
  col       max |u_n - v_n| over the columns of non-degenerate eigenvalues (with
            --eigenvalues): phase-fixed vectors of a simple eigenvalue agree
            entry by entry

Usage: python -m laph_eigsys_b200.compare DIR_U DIR_V --conf N --lx L --nev K [--timeslices 0 1 ...]
       [--eigenvalues] (also read eigenvalues.%04d.%03d from both) [--json]
Host-only: numpy and the library's file readers (no device)."""
import argparse
import json
import sys

import numpy as np

from . import read_eigenvalues_bin, read_eigsys_bin


def cluster_ends(lam, nev, gap):
    """End indices (exclusive) of the clusters of sorted eigenvalues lam[0..) that lie wholly inside the first nev;
    a cluster whose last member is the nev-th and whose next eigenvalue is unknown counts as complete."""
    ends = []
    i = 0
    while i < nev:
        j = i + 1
        while j < nev and lam[j] - lam[j - 1] < gap:
            j += 1
        if j < nev or len(lam) <= nev or lam[nev] - lam[nev - 1] >= gap:
            ends.append(j)
        i = j
    return ends


def compare_timeslice(U, V, lam_u=None, lam_v=None, gap=1e-6 * 12.0):
    """Numbers for one timeslice; U, V column-major [3 V3][nev] blocks, lam_* the stored eigenvalues (<= 0)."""
    N = U.conj().T @ V
    out = {"tr_uv": complex(np.trace(N)), "sum_uv": complex(N.sum()), "sum_abs2_uv": float((np.abs(N) ** 2).sum()),
           "tr_uu": float(np.trace(U.conj().T @ U).real), "tr_vv": float(np.trace(V.conj().T @ V).real),
           "phase": float(max(np.abs(np.angle(U[0])).max(), np.abs(np.angle(V[0])).max()))}
    nev = U.shape[1]
    if lam_u is not None and lam_v is not None:
        lu, lv = -np.asarray(lam_u), -np.asarray(lam_v)
        out["dlam"] = float(np.abs(lu - lv).max() / 12.0)
        # subspace distance per complete cluster of the sorted spectrum, from the principal angles
        order_u, order_v = np.argsort(lu), np.argsort(lv)
        ends = cluster_ends(lu[order_u], nev, gap)
        worst = 0.0
        for end in ends:  # the span of the first `end` eigenvectors is unique when `end` closes a cluster
            worst = max(worst, sin_max_angle(U[:, order_u[:end]], V[:, order_v[:end]]))
        out["proj"] = worst
        out["clusters_checked"] = len(ends)
        col, start = 0.0, 0
        for end in ends:
            if end - start == 1:  # a simple eigenvalue: the phase-fixed vector is unique
                col = max(col, float(np.abs(U[:, order_u[start]] - V[:, order_v[start]]).max()))
            start = end
        out["col"] = col
    else:
        out["proj"] = sin_max_angle(U, V)
    return out


def sin_max_angle(A, B):
    """sin of the largest principal angle between span(A) and span(B) (orthonormal columns) = ||A A^dag - B B^dag||_2,
    as ||(1 - A A^dag) B||_2: no cancellation when the subspaces agree (1 - cos^2 would lose half the digits)."""
    M = B - A @ (A.conj().T @ B)
    return float(np.sqrt(max(0.0, np.linalg.eigvalsh(M.conj().T @ M).max())))


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m laph_eigsys_b200.compare", description=__doc__.splitlines()[0])
    ap.add_argument("dir_u")
    ap.add_argument("dir_v")
    ap.add_argument("--conf", type=int, required=True)
    ap.add_argument("--lx", type=int, required=True)
    ap.add_argument("--nev", type=int, required=True)
    ap.add_argument("--timeslices", type=int, nargs="+", default=[0])
    ap.add_argument("--eigenvalues", action="store_true")
    ap.add_argument("--json", action="store_true")
    a = ap.parse_args(argv)
    dim = 3 * a.lx ** 3
    worst = {"dlam": 0.0, "proj": 0.0, "col": 0.0}
    for t in a.timeslices:
        U = read_eigsys_bin(a.dir_u, "eigenvectors", a.conf, t, dim, a.nev)
        V = read_eigsys_bin(a.dir_v, "eigenvectors", a.conf, t, dim, a.nev)
        lu = lv = None
        if a.eigenvalues:
            lu = read_eigenvalues_bin(a.dir_u, "eigenvalues", a.conf, t, a.nev)
            lv = read_eigenvalues_bin(a.dir_v, "eigenvalues", a.conf, t, a.nev)
        r = compare_timeslice(U, V, lu, lv)
        for k in worst:
            if k in r:
                worst[k] = max(worst[k], r[k])
        if a.json:
            print(json.dumps({"t": t, **{k: (str(v) if isinstance(v, complex) else v) for k, v in r.items()}}))
        else:
            print(f"ts {t}: tr(U^dag V) = {r['tr_uv']:.12g}  sum(U^dag V) = {r['sum_uv']:.6g}  "
                  f"sum|U^dag V|^2 = {r['sum_abs2_uv']:.12g}  tr(U^dag U) = {r['tr_uu']:.12g}  "
                  f"tr(V^dag V) = {r['tr_vv']:.12g}  proj = {r['proj']:.3e}"
                  + (f"  dlam = {r['dlam']:.3e}  col = {r['col']:.3e}" if "dlam" in r else ""))
    print(json.dumps({"worst": worst}) if a.json else f"worst: {worst}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
