"""CPU, two ranks over gloo: the host logic of `bench.py --gpus N`.

Multi-GPU runs are replicas: every rank solves its own seeded cell, and no
collective is on the data path. The job's figures reduce per-rank numbers
over the ranks. The units add up, and the time is the slowest rank's. These
tests run that reduction with torch.distributed on the gloo backend, two
processes on 127.0.0.1. They also check that the ranks' seeded decks
differ, so the replicas are independent cells and not one cell twice.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r processed 1e9 (r + 1) updates in 0.5 (r + 1) s
        rate = bench.whole_job_rate(1e9 * (rank + 1), 0.5 * (rank + 1), world, "cpu")
        mx = bench.ranks_reduce(3.0 + rank, "max", world, "cpu")
        sm = bench.ranks_reduce(3.0 + rank, "sum", world, "cpu")
        deck, _ = bench.build_deck("config2", seed=rank)
        out[rank] = (rate, mx, sm, deck.mesh.n_cells, float(deck.mesh.nodes[:, 0].sum()))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(600)
def test_two_ranks_reduce_like_the_bench():
    world = 2
    with mp.get_context("spawn").Manager() as man:
        out = man.dict()
        mp.start_processes(_rank_main, args=(world, free_port(), out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    # (1e9 + 2e9) updates over the slowest rank's 1.0 s, on every rank
    for r in range(world):
        rate, mx, sm, _, _ = res[r]
        assert rate == pytest.approx(3e9)
        assert mx == 4.0 and sm == 7.0
    # independent seeded cells: different meshes on the two ranks
    assert (res[0][3], res[0][4]) != (res[1][3], res[1][4])


def test_one_rank_is_the_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.ranks_reduce(2.5, "max", 1, "cpu") == 2.5
    assert bench.whole_job_rate(10.0, 4.0, 1, "cpu") == 2.5
