#!/usr/bin/env python3
"""Generates tests/golden/*.npz: seeded inputs and the CPU FP64 oracle's
outputs for them, plus analytic known answers.  The reference ships no
golden data and cannot be built here, so these pin the oracle's and the CUDA
path's results against regressions; the analytic parts (free spectrum) pin
them against the mathematics.  Run from the repository root:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import laph_eigsys_b200 as lb  # noqa: E402
import oracle as orc  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def main():
    L = 4
    conf = lb.gauge_random(L, 2, 0.4, 1227)
    U = np.ascontiguousarray(conf[0, :, 1:4])
    smeared = {
        "stout_compat": orc.smear_stout(U, L, 0.1, 3, 1),
        "stout": orc.smear_stout(U, L, 0.1, 3, 0),
        "ape_compat": orc.smear_ape(U, L, 0.5, 3, 1),
        "hyp": orc.smear_hyp(U, L, 0.62, 0.52, 3),
    }
    Us = smeared["hyp"]
    w = np.linalg.eigvalsh(orc.neglap_dense(Us, L))
    rng = np.random.default_rng(1227)
    x = rng.normal(size=3 * L ** 3) + 1j * rng.normal(size=3 * L ** 3)
    y8 = orc.tv_iter(Us, L, 11.8, 0.6, 8, x)
    np.savez_compressed(os.path.join(OUT, "l4_seed1227.npz"), conf=conf, x=x, tv_iter_deg8_hyp=y8,
                        neglap_eigs_hyp=w, plaquette_hyp=orc.plaquette(Us, L), **smeared)
    # the eigensystem's consumers on a stored block: the 6 lowest eigenvectors of the HYP-smeared -Delta
    # (numpy's eigh, stored as input, so nothing depends on its phase or degenerate-subspace choices),
    # the source shape psi(r) with its radius average, and the covariant displacement along x, y, z
    _, Vall = np.linalg.eigh(orc.neglap_dense(Us, L))
    V = np.asfortranarray(Vall[:, :6])
    psi = orc.sourceshape(V, L)
    r, avg = orc.sourceshape_avg(L, psi)
    W = np.stack([orc.displace(Us, L, d, V) for d in range(3)])
    np.savez_compressed(os.path.join(OUT, "l4_hyp_consumers.npz"), V=V, psi=psi, radii=r, psi_avg=avg, displaced=W)
    np.savez_compressed(os.path.join(OUT, "free_spectrum.npz"), L4=orc.free_spectrum(4), L6=orc.free_spectrum(6),
                        L8=orc.free_spectrum(8))
    print("wrote", sorted(f for f in os.listdir(OUT) if f.endswith(".npz")))


if __name__ == "__main__":
    main()
