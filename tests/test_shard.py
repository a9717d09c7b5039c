"""CPU: the host side of direction sharding (giftbte_b200.shard).

The block partition follows the reference's count of local directions per
rank; the exchanges sum buffers in place. The thread exchange runs here on
host buffers; the torch.distributed exchange runs as two gloo ranks on
127.0.0.1, called through a C function pointer of the ABI's
gbte_exchange_fn type, as the library calls it.
"""
import os
import socket
import sys
import threading

import numpy as np
import pytest
import torch.multiprocessing as mp

from giftbte_b200 import EXCHANGE_FN, shard

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("nd,parts", [(64, 1), (64, 2), (64, 3), (64, 8), (32, 5), (128, 7), (4, 4)])
def test_blocks_cover_the_directions_once(nd, parts):
    bl = shard.direction_blocks(nd, parts)
    assert len(bl) == parts
    assert bl[0][0] == 0
    for (b0, n0), (b1, _) in zip(bl, bl[1:]):
        assert b1 == b0 + n0
    assert sum(n for _, n in bl) == nd
    # nd // parts each, one more for the first nd % parts blocks
    assert [n for _, n in bl] == [nd // parts + (1 if r < nd % parts else 0) for r in range(parts)]


def test_blocks_reject_empty_parts():
    with pytest.raises(ValueError):
        shard.direction_blocks(4, 5)
    with pytest.raises(ValueError):
        shard.direction_blocks(4, 0)


def run_members(x, bufs, rounds=1):
    errs = [None] * len(bufs)

    def run(k):
        try:
            fn = x.member(k, device="cpu")
            for _ in range(rounds):
                fn(bufs[k].ctypes.data, bufs[k].size, 0)
        except BaseException as e:
            errs[k] = e
            x.abort()

    ts = [threading.Thread(target=run, args=(k,)) for k in range(len(bufs))]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    return errs


def test_thread_exchange_sums_in_handle_order():
    rng = np.random.default_rng(0)
    src = [rng.standard_normal(1001) for _ in range(3)]
    bufs = [s.copy() for s in src]
    x = shard.ThreadExchange(3, timeout=30.0)
    assert run_members(x, bufs) == [None] * 3
    want = (src[0] + src[1]) + src[2]
    for b in bufs:
        assert np.array_equal(b, want)
    assert x.calls == 1


def test_thread_exchange_union_of_zeroed_blocks_is_exact():
    # each member holds its block and zeros elsewhere, as the solver's
    # boundary values and margins are exchanged: the sum is the union, bit for bit
    rng = np.random.default_rng(1)
    full = rng.standard_normal(12 * 7)
    bufs = []
    for b, n in shard.direction_blocks(12, 3):
        v = np.zeros_like(full)
        v[b * 7:(b + n) * 7] = full[b * 7:(b + n) * 7]
        bufs.append(v)
    x = shard.ThreadExchange(3, timeout=30.0)
    assert run_members(x, bufs, rounds=1) == [None] * 3
    for v in bufs:
        assert np.array_equal(v, full)


def test_thread_exchange_failure_breaks_every_member():
    x = shard.ThreadExchange(2, timeout=30.0)
    bufs = [np.ones(4), np.ones(5)]  # different sizes: member 0 refuses the sum
    errs = run_members(x, bufs)
    assert isinstance(errs[0], RuntimeError)
    assert isinstance(errs[1], threading.BrokenBarrierError)


def test_exchange_fn_pointer_round_trip():
    # a Python exchange behind the ABI's function-pointer type, called the
    # way the library calls it
    seen = {}

    def cb(user, buf, n, stream):
        shard.host_doubles(buf, n)[:] *= 2.0
        seen["args"] = (user, n, stream)
        return 0

    fp = EXCHANGE_FN(cb)
    a = np.arange(6, dtype=np.float64)
    assert fp(None, a.ctypes.data, a.size, None) == 0
    assert np.array_equal(a, 2.0 * np.arange(6))
    assert seen["args"] == (None, 6, None)


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    from giftbte_b200 import EXCHANGE_FN as FN
    from giftbte_b200 import shard as sh

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ex = sh.torch_exchange(device="cpu")

        def cb(user, buf, n, stream):
            ex(buf, int(n), stream or 0)
            return 0

        fp = FN(cb)
        nd, w = 10, 3
        full = np.arange(nd * w, dtype=np.float64) + 0.5
        b, n = sh.direction_blocks(nd, world)[rank]
        buf = np.zeros(nd * w)
        buf[b * w:(b + n) * w] = full[b * w:(b + n) * w]
        rc = fp(None, buf.ctypes.data, buf.size, None)
        # margins: only the rank holding direction 0 contributes
        marg = np.array([3.0, 4.0, 5.0, 6.0]) if b == 0 else np.zeros(4)
        rc2 = fp(None, marg.ctypes.data, marg.size, None)
        out[rank] = (rc, rc2, buf.tolist(), marg.tolist(), full.tolist())
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(600)
def test_two_gloo_ranks_exchange_through_the_function_pointer():
    world = 2
    with mp.get_context("spawn").Manager() as man:
        out = man.dict()
        mp.start_processes(_rank_main, args=(world, free_port(), out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    for r in range(world):
        rc, rc2, buf, marg, full = res[r]
        assert rc == 0 and rc2 == 0
        assert buf == full
        assert marg == [3.0, 4.0, 5.0, 6.0]
