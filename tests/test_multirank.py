"""Multi-process path on CPU (gloo, world size 2): timeslices are split across
ranks as the reference splits them across MPI ranks (src/ev_ts.cpp:103-119),
each rank reads only its slab of the LIME file, and the gathered slabs
reproduce the whole configuration -- no collective on the data path, one
all_gather of a checksum for the check."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import laph_eigsys_b200 as lb


def test_split_matches_reference_rule():
    for LT, size in [(48, 7), (64, 8), (16, 3), (5, 8), (96, 1)]:
        blocks = [lb.timeslice_split(LT, size, r) for r in range(size)]
        assert sum(n for _, n in blocks) == LT
        t = 0
        for r, (t0, n) in enumerate(blocks):
            assert t0 == t and n == LT // size + (1 if r < LT % size else 0)
            t += n


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, path, L, T, out):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    t0, n = lb.timeslice_split(T, world, rank)
    conf = lb.lime_read_gauge(path, T, L, t0, t0 + n - 1)
    mine = torch.tensor([float(t0), float(n), float(np.abs(conf).sum()), float(conf.real.sum())],
                        dtype=torch.float64)
    got = [torch.zeros(4, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(got, mine)
    if rank == 0:
        np.save(out, torch.stack(got).numpy())
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_two_ranks_read_their_slabs(tmp_path, world):
    L, T = 4, 7
    conf = lb.gauge_random(L, T, 0.4, 321)
    path = tmp_path / "conf.0001"
    lb.lime_write_gauge(path, conf, L, T)
    out = str(tmp_path / "gathered.npy")
    mp.start_processes(_rank_main, args=(world, _free_port(), str(path), L, T, out), nprocs=world, join=True,
                       start_method="spawn")
    got = np.load(out)
    assert got[:, 1].sum() == T and got[0, 0] == 0 and got[1, 0] == got[0, 1]
    assert abs(got[:, 2].sum() - np.abs(conf).sum()) < 1e-9 * np.abs(conf).sum()
    assert abs(got[:, 3].sum() - conf.real.sum()) < 1e-9
