#!/usr/bin/env python3
"""Train the learned Chebyshev window (laph_eigsys_b200/data/window_mlp.bin).

Windows come from the non-learned block solver (window = LAPH_WINDOW_LANCZOS)
run on seeded synthetic lattices (seeds 2000+, 16^3 to 32^3, several
roughnesses, smearings and nev); the network is trained on the GPU by the
library's own forward / backward / Adam kernels.  Usage:

    python -m laph_eigsys_b200.train_window [--quick] [--out PATH]
"""
import argparse
import json
import os
import sys
import time

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import laph_eigsys_b200 as lb  # noqa: E402
from laph_eigsys_b200 import window  # noqa: E402

SMEARS = [("stout", lb.SMEAR_STOUT, 0.1, 0.0, 3), ("stout", lb.SMEAR_STOUT, 0.1, 0.0, 6),
          ("hyp", lb.SMEAR_HYP, 0.62, 0.62, 1), ("hyp", lb.SMEAR_HYP, 0.62, 0.52, 3),
          ("ape", lb.SMEAR_APE, 0.5, 0.0, 10), ("none", lb.SMEAR_NONE, 0.0, 0.0, 0)]


def plan(quick):
    seed = 2000
    runs = []
    eps_list = [0.2, 0.3, 0.4] if quick else [0.2, 0.25, 0.3, 0.35, 0.4, 0.45]
    for eps in eps_list:
        for sm in SMEARS:
            for nev in ([60] if quick else [40, 60, 80]):
                runs.append(dict(L=16, T=16 if quick else 64, nev=nev, eps=eps, smear=sm, seed=seed))
                seed += 1
    if not quick:
        for eps in [0.25, 0.3, 0.35, 0.4]:
            for sm in SMEARS[:5]:
                runs.append(dict(L=24, T=32, nev=120, eps=eps, smear=sm, seed=seed))
                seed += 1
        for eps in [0.25, 0.3, 0.35]:
            for sm in SMEARS[:3]:
                runs.append(dict(L=32, T=16, nev=120, eps=eps, smear=sm, seed=seed))
                seed += 1
    return runs


def solve_windows(r, device):
    L, T, nev = r["L"], r["T"], r["nev"]
    name, kind, p1, p2, it = r["smear"]
    conf = lb.gauge_random(L, T, r["eps"], r["seed"])
    s = lb.Solver([(L, nev)] * T, device=device, smear_kind=kind, smear_p1=p1, smear_p2=p2, smear_iters=it,
                  smear_compat=1, guard=16, link_prec=lb.LINKS_FP32, tol=1e-9, max_it=300, deg=48,
                  window=lb.WINDOW_LANCZOS)
    for t in range(T):
        s.set_links(t, conf[t], lb.LAYOUT_CONF)
    st, res = s.run()
    X, Y = window.collect(s)
    ok = np.array([q["status"] == 0 for q in res])
    iters = [q["iters"] for q in res]
    s.close()
    return X[ok], Y[ok], iters


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--out", default=window.MODEL_PATH)
    ap.add_argument("--epochs", type=int, default=4000)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()
    t0 = time.time()
    Xs, Ys = [], []
    for r in plan(args.quick):
        X, Y, iters = solve_windows(r, args.device)
        Xs.append(X)
        Ys.append(Y)
        print(json.dumps({"L": r["L"], "nev": r["nev"], "eps": r["eps"], "smear": r["smear"][0], "n": len(X),
                          "mean_iters": float(np.mean(iters))}), flush=True)
    X, Y = np.concatenate(Xs), np.concatenate(Ys)
    rng = np.random.default_rng(0)
    perm = rng.permutation(len(X))
    nval = max(1, len(X) // 10)
    val, tr = perm[:nval], perm[nval:]
    model, loss = window.train(X[tr], Y[tr], epochs=args.epochs, device=args.device)
    pred = window.predict(model, X[val], device=args.device)
    rmse = np.sqrt(((pred - Y[val]) ** 2).mean(0))
    rel_cut = np.abs(np.exp(pred[:, 0]) - np.exp(Y[val, 0])) / np.exp(Y[val, 0])
    report = {"windows": int(len(X)), "train": int(len(tr)), "val": int(nval), "train_loss_std": loss,
              "val_rmse": rmse.tolist(), "val_cut_rel_err_median": float(np.median(rel_cut)),
              "val_cut_rel_err_p90": float(np.quantile(rel_cut, 0.9)), "seconds": time.time() - t0}
    window.save_model(model, args.out, meta=json.dumps(report).encode())
    print(json.dumps(report), flush=True)
    np.savez_compressed(os.path.splitext(args.out)[0] + "_data.npz", X=X, Y=Y)


if __name__ == "__main__":
    main()
