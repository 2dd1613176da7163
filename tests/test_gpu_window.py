"""Learned Chebyshev window: the device MLP kernels against the FP64 CPU
oracle (forward, gradient), training reduces the loss, and the ablation --
the trained network's first window against the non-learned method on
timeslices it was not trained on: both reach the tolerance, with the same
spectrum, and the learned window needs strictly fewer outer iterations and
less solve time.  A window that fails its check after the first pass falls
back to the non-learned one and still converges."""
import os

import numpy as np
import pytest

from conftest import random_links

pytestmark = pytest.mark.gpu


def test_mlp_gradient_matches_oracle(gpu, orc):
    from laph_eigsys_b200 import window
    rng = np.random.default_rng(3)
    P = window.init_params(7) + rng.normal(scale=0.05, size=window.NPARAMS).astype(np.float32)
    X = rng.normal(size=(37, 16)).astype(np.float32)
    Y = rng.normal(size=(37, 3)).astype(np.float32)
    loss, g = window.grad(P, X, Y)
    loss_ref, g_ref = orc.mlp_loss_grad(P.astype(np.float64), X.astype(np.float64), Y.astype(np.float64))
    assert abs(loss - loss_ref) / loss_ref < 1e-5
    assert np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref) < 1e-4


def test_mlp_forward_matches_numpy(gpu):
    from laph_eigsys_b200 import window
    rng = np.random.default_rng(4)
    P = window.init_params(1).astype(np.float64)
    X = rng.normal(size=(20, 16))
    W1 = P[:1024].reshape(64, 16); b1 = P[1024:1088]
    W2 = P[1088:5184].reshape(64, 64); b2 = P[5184:5248]
    W3 = P[5248:5440].reshape(3, 64); b3 = P[5440:5443]
    ref = np.tanh(np.tanh(X @ W1.T + b1) @ W2.T + b2) @ W3.T + b3
    model = np.concatenate([P, np.zeros(16), np.ones(16), np.zeros(3), np.ones(3)]).astype(np.float32)
    out = window.predict(model, X.astype(np.float32))
    assert np.abs(out - ref).max() < 1e-5


def test_mlp_training_reduces_loss(gpu):
    from laph_eigsys_b200 import window
    rng = np.random.default_rng(5)
    X = rng.normal(size=(400, 16)).astype(np.float32)
    Y = np.stack([np.sin(X[:, 0]) + X[:, 1] ** 2, X[:, 2] * X[:, 3], np.tanh(X[:, 4])], 1).astype(np.float32)
    P = window.init_params(0)
    l0, _ = window.grad(P, (X - X.mean(0)) / X.std(0), (Y - Y.mean(0)) / Y.std(0))
    model, l1 = window.train(X, Y, epochs=600, lr=3e-3)
    assert l1 < 0.15 * l0


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                                    "laph_eigsys_b200", "data", "window_mlp.bin")),
                    reason="window model not trained yet")
def test_learned_window_ablation(gpu):
    from laph_eigsys_b200 import window
    model = window.load_model()
    L, T, nev = 16, 16, 60
    conf = gpu.gauge_random(L, T, 0.3, 1230)  # the 16^3 lattice seed of the mixed-volume workload, not a training seed
    out = {}
    for mode in (gpu.WINDOW_LANCZOS, gpu.WINDOW_MLP):
        s = gpu.Solver([(L, nev)] * T, smear_kind=gpu.SMEAR_APE, smear_p1=0.5, smear_iters=10, guard=16,
                       tol=1e-9, deg=48, window=mode, link_prec=gpu.LINKS_FP32)
        if mode == gpu.WINDOW_MLP:
            window.set_model(s, model)
        for t in range(T):
            s.set_links(t, conf[t], gpu.LAYOUT_CONF)
        st, res = s.run()
        assert st == 0
        out[mode] = ([r["iters"] for r in res], [s.get(t, vectors=False)[0] for t in range(T)], s.timings()[3])
        s.close()
    it_l, ev_l, ms_l = out[gpu.WINDOW_LANCZOS]
    it_m, ev_m, ms_m = out[gpu.WINDOW_MLP]
    for a, b in zip(ev_l, ev_m):
        assert np.abs(a - b).max() <= 2e-9 * 12
    print(f"outer iterations: lanczos window {max(it_l)}, learned window {max(it_m)}; "
          f"batch ms {ms_l:.1f} -> {ms_m:.1f}")
    assert max(it_m) < max(it_l)
    assert ms_m < ms_l


def test_learned_window_fallback(gpu, orc):
    """A model whose first window is far off -- its cut a hundred times too low, so the first pass amplifies almost
    nothing -- fails the check after the first pass; the solve falls back to the non-learned window, says so in
    window_fallback, and still returns the dense spectrum."""
    from laph_eigsys_b200 import window
    model = window.load_model()
    L, nev, T = 8, 20, 4
    links = [random_links(L, 0.4, 1231 + t) for t in range(T)]
    s = gpu.Solver([(L, nev)] * T, smear_kind=gpu.SMEAR_NONE, guard=12, tol=1e-10, deg=32, window=gpu.WINDOW_MLP,
                   window_margin=0.01, link_prec=gpu.LINKS_FP32)
    window.set_model(s, model)
    for t, U in enumerate(links):
        s.set_links(t, U)
    st, res = s.run()
    assert st == 0
    print("fallbacks", [r["window_fallback"] for r in res])
    assert sum(r["window_fallback"] for r in res) >= 1
    for t, U in enumerate(links):
        ev, V, _ = s.get(t)
        w = np.linalg.eigvalsh(orc.neglap_dense(U, L))[:nev]
        assert np.abs(-ev - w).max() <= 1e-9 * 12
    s.close()
