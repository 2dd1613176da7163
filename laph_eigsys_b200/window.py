"""Learned Chebyshev window: data, training and the model file.

The block solver's first filter pass needs a damped interval [lambda_cut,
lambda_max] and a degree before any Ritz value exists.  A 16 -> 64 -> 64 -> 3
MLP (FP32, trained and evaluated by this library's own CUDA kernels) maps
per-timeslice features -- smeared-plaquette moments and the Ritz values of a
10-step Lanczos, computed on the device by the solver -- to

    target 0: log of the window cut the non-learned (Lanczos/adaptive) solver
              converges to, i.e. its final largest Ritz value theta_{k-1};
    target 1: lambda_max (the 10-step Lanczos upper bound; reported only: the
              solver keeps the exact bound 12 of the spectrum of -Delta);
    target 2: a filter degree: the smallest m that damps the slowest wanted
              pair theta_{nev-1} relative to theta_{k-1} by FIRST_PASS_GAIN.

Training windows come from solves of the non-learned method itself
(window = LAPH_WINDOW_LANCZOS) on seeded synthetic lattices; that solver's
residual check is what judges every window, learned or not.
"""
import ctypes
import os
import struct

import numpy as np

from . import _lib
from ._lib import check, lib

NPARAMS = lib.laph_mlp_nparams()
NIN, NH, NOUT = 16, 64, 3
NNORM = 2 * NIN + 2 * NOUT
MODEL_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "window_mlp.bin")
MAGIC = b"LAPHMLP1"
FIRST_PASS_GAIN = 10.0 ** 1.5


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def init_params(seed=0):
    """Glorot-uniform weights, zero biases, in the library's parameter layout."""
    rng = np.random.default_rng(seed)
    parts = []
    for fan_out, fan_in in [(NH, NIN), (NH, NH), (NOUT, NH)]:
        a = np.sqrt(6.0 / (fan_in + fan_out))
        parts += [rng.uniform(-a, a, size=fan_out * fan_in), np.zeros(fan_out)]
    p = np.concatenate(parts).astype(np.float32)
    assert p.size == NPARAMS
    return p


def degree_target(theta, nev, lam_max=12.0, lo=16, hi=64):
    """Smallest degree with T_m(theta_B(theta_{nev-1})) >= FIRST_PASS_GAIN for the
    window [theta_{k-1}, lam_max] (theta ascending, length k)."""
    cut = theta[-1]
    tb = 1.0 + 2.0 * (cut - theta[nev - 1]) / (lam_max - cut)
    m = np.arccosh(FIRST_PASS_GAIN) / np.arccosh(max(tb, 1.0 + 1e-9))
    return float(np.clip(np.ceil(m), lo, hi))


def collect(solver):
    """(features [n,16], targets [n,3]) from a solver that ran with the non-learned window."""
    n = len(solver.problems)
    feats = np.empty((n, NIN), dtype=np.float32)
    bound = np.empty(n)
    check(lib.laph_solver_features(solver._h, _p(feats), _p(bound)), "laph_solver_features")
    Y = np.empty((n, NOUT), dtype=np.float32)
    for i, (L, nev) in enumerate(solver.problems):
        kmax = 512
        th = np.empty(kmax)
        k = ctypes.c_int()
        check(lib.laph_solver_ritz(solver._h, i, _p(th), ctypes.byref(k)), "laph_solver_ritz")
        th = np.sort(th[:k.value])
        Y[i] = [np.log(th[-1]), bound[i], degree_target(th, nev)]
    return feats, Y


def train(X, Y, epochs=4000, lr=3e-3, seed=0, device=0):
    """Standardise, train with full-batch Adam on the device; returns (model, final loss)."""
    X = np.asarray(X, dtype=np.float32)
    Y = np.asarray(Y, dtype=np.float32)
    xm, xs = X.mean(0), X.std(0) + 1e-12
    ym, ys = Y.mean(0), Y.std(0) + 1e-12
    Xn = np.ascontiguousarray((X - xm) / xs, dtype=np.float32)
    Yn = np.ascontiguousarray((Y - ym) / ys, dtype=np.float32)
    params = init_params(seed)
    loss = ctypes.c_float()
    check(lib.laph_mlp_train(_p(params), _p(Xn), _p(Yn), Xn.shape[0], epochs, lr, ctypes.byref(loss), device),
          "laph_mlp_train")
    model = np.concatenate([params, xm, xs, ym, ys]).astype(np.float32)
    return model, float(loss.value)


def predict(model, X, device=0):
    """Targets predicted by a model for raw features X [n,16]."""
    X = np.asarray(X, dtype=np.float32)
    params = np.ascontiguousarray(model[:NPARAMS])
    xm, xs = model[NPARAMS:NPARAMS + NIN], model[NPARAMS + NIN:NPARAMS + 2 * NIN]
    ym, ys = model[NPARAMS + 2 * NIN:NPARAMS + 2 * NIN + NOUT], model[NPARAMS + 2 * NIN + NOUT:]
    Xn = np.ascontiguousarray((X - xm) / xs, dtype=np.float32)
    out = np.empty((X.shape[0], NOUT), dtype=np.float32)
    check(lib.laph_mlp_forward(_p(params), _p(Xn), X.shape[0], _p(out), device), "laph_mlp_forward")
    return out * ys + ym


def save_model(model, path=MODEL_PATH, meta=b""):
    model = np.ascontiguousarray(model, dtype=np.float32)
    assert model.size == NPARAMS + NNORM
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "wb") as f:
        f.write(MAGIC + struct.pack("<ii", NPARAMS, NNORM))
        f.write(model.tobytes())
        f.write(meta)


def load_model(path=MODEL_PATH):
    with open(path, "rb") as f:
        head = f.read(16)
        if head[:8] != MAGIC:
            raise ValueError(f"{path}: not a window model")
        npar, nnorm = struct.unpack("<ii", head[8:16])
        if npar != NPARAMS or nnorm != NNORM:
            raise ValueError(f"{path}: model of another shape")
        return np.frombuffer(f.read(4 * (npar + nnorm)), dtype=np.float32).copy()


def set_model(solver, model):
    model = np.ascontiguousarray(model, dtype=np.float32)
    check(lib.laph_solver_set_window_model(solver._h, _p(model), model.size), "laph_solver_set_window_model")


def grad(params, X, Y, device=0):
    """Loss and gradient of the mean-squared loss from the device kernels."""
    params = np.ascontiguousarray(params, dtype=np.float32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    Y = np.ascontiguousarray(Y, dtype=np.float32)
    g = np.empty(NPARAMS, dtype=np.float32)
    loss = ctypes.c_float()
    check(lib.laph_mlp_grad(_p(params), _p(X), _p(Y), X.shape[0], _p(g), ctypes.byref(loss), device),
          "laph_mlp_grad")
    return float(loss.value), g
