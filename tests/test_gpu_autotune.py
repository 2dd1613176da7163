"""laph_solver_autotune on the device: the chosen settings come from the
candidate lists, the cache file records them and a second call reads them back
without timing anything, and a solve with the tuned settings matches a dense
FP64 eigendecomposition of the oracle's assembled -Delta."""
import numpy as np
import pytest

from conftest import random_links

pytestmark = pytest.mark.gpu


def test_autotune_picks_cached_settings_that_solve_correctly(gpu, orc, tmp_path):
    L, nev = 8, 20
    links = [random_links(L, 0.4, 70 + i) for i in range(3)]
    probs = [(L, nev)] * 3
    cache = tmp_path / "tune.txt"
    kw = dict(tol=1e-10, deg=60, max_it=300, guard=16, window=gpu.WINDOW_LANCZOS, link_prec=gpu.LINKS_FP32)
    opts, r = gpu.autotune(probs, links, nsample=2, cache=cache, **kw)
    # deg (8) + block (3 more) + guard (up to 2 more) + tile (2 more)
    assert r["from_cache"] == 0 and 1 <= r["trials"] <= 15 and r["ms_per_problem"] > 0
    # nev 20: guard 16 (k 64), 48 (k 96), 12 (k 32)
    assert r["deg"] in (40, 48, 56, 60, 64, 72, 80, 96) and r["block"] in (8, 16, 32, 64) and r["guard"] in (16, 48, 12)
    assert r["tile"] in (64, 128, 256)
    assert (opts.deg, opts.block, opts.guard, opts.filter_tile) == (r["deg"], r["block"], r["guard"], r["tile"])
    lines = cache.read_text().splitlines()
    assert len(lines) == 1 and lines[0].split("\t")[1].split()[:3] == [str(r["deg"]), str(r["block"]), str(r["guard"])]
    opts2, r2 = gpu.autotune(probs, links, nsample=2, cache=cache, **kw)
    assert r2["from_cache"] == 1 and r2["trials"] == 0
    assert (r2["deg"], r2["block"], r2["guard"], r2["tile"]) == (r["deg"], r["block"], r["guard"], r["tile"])
    s = gpu.Solver(probs, opts=opts)
    for i in range(3):
        s.set_links(i, links[i])
    st, res = s.run()
    assert st == 0
    for i in range(3):
        ev, V, _ = s.get(i)
        w = np.linalg.eigvalsh(orc.neglap_dense(links[i], L))
        assert np.abs(-ev - w[:nev]).max() / w[-1] <= 1e-10
        assert np.abs(V.conj().T @ V - np.eye(nev)).max() <= 1e-10
    s.close()


def test_footprint_matches_device_allocation(gpu):
    """laph_solver_footprint against the free-memory drop of an actual laph_solver_create (two 32^3 timeslices,
    about 2.7 GB): within the 2 MiB-per-allocation rounding it assumes; laph_solver_max_batch fits them."""
    import torch
    probs = [(32, 120)] * 2
    kw = dict(guard=16, deg=60, link_prec=gpu.LINKS_FP32)
    fp = gpu.solver_footprint(probs, **kw)
    assert gpu.solver_max_batch(probs, **kw) == 2
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    s = gpu.Solver(probs, **kw)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    used = free0 - free1
    s.close()
    assert 0.85 * fp <= used <= 1.02 * fp + (64 << 20), (used, fp)
