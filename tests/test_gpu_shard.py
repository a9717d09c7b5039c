"""GPU: direction sharding of one solve (gbte_set_direction_shard).

The handles of a shard set share the one GPU here, one host thread each,
and exchange through ``giftbte_b200.shard.ThreadExchange`` (a host barrier
and a sum in handle order; no kernel waits on another handle's kernels).
The sharded solve must reach the whole solve's fixed point: on the golden
decks, against the compiled reference's fields at 1e-9, as the whole solve
does, with specular walls whose reflected directions sit in another block.
"""
import numpy as np
import pytest

import giftbte_b200 as g
import make_golden as mg
from giftbte_b200 import decks, shard

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def solve_sharded(deck, parts, prec, T0=None, **solve_kw):
    hs = [g.StaticBTESynthetic.from_deck(deck, precision=prec) for _ in range(parts)]
    x = shard.ThreadExchange(parts, timeout=120.0)
    for k, (b, n) in enumerate(shard.direction_blocks(hs[0].num_directions, parts)):
        hs[k].set_direction_shard(b, n, x.member(k))
    for h in hs:
        if T0 is None:
            h.fourier_initial()
        else:
            h.set_initial(T0)
    sts = shard.solve_sharded(hs, x, **solve_kw)
    fs = [h.fields() for h in hs]
    for h in hs:
        h.close()
    return fs, sts, x.calls


def solve_whole(deck, prec, T0=None, **solve_kw):
    s = g.StaticBTESynthetic.from_deck(deck, precision=prec)
    if T0 is None:
        s.fourier_initial()
    else:
        s.set_initial(T0)
    st = s.solve(**solve_kw)
    f = s.fields()
    s.close()
    return f, st


def test_one_block_is_the_whole_solve_bit_for_bit():
    # a shard set of one handle: the exchange sums one buffer, the
    # transport runs as two graphs around it
    deck, ref = mg.load("porous_msh")
    fw, sw = solve_whole(deck, g.GBTE_FP64, ref["Tf"], max_iter=40, err_temp=0.0, err_flux=0.0)
    fs, ss, calls = solve_sharded(deck, 1, g.GBTE_FP64, ref["Tf"], max_iter=40, err_temp=0.0, err_flux=0.0)
    for k in ("T", "E", "q", "Tband"):
        assert np.array_equal(fw[k], fs[0][k]), k
    assert ss[0]["iterations"] == sw["iterations"] == 40
    assert calls == 2 * 40  # moments and margins, every outer iteration


@pytest.mark.parametrize("case", ["porous_msh", "quad_heat_specular", "periodic_jitter", "gray_square_tri"])
@pytest.mark.parametrize("parts", [2, 3])
def test_shards_reach_the_reference_fixed_point(case, parts):
    deck, ref = mg.load(case)
    fw, sw = solve_whole(deck, g.GBTE_FP64, ref["Tf"], allow_not_converged=False)
    fs, ss, _ = solve_sharded(deck, parts, g.GBTE_FP64, ref["Tf"], allow_not_converged=False)
    # every handle stops at the same iteration and holds the whole fields
    assert len({s["iterations"] for s in ss}) == 1
    assert abs(ss[0]["iterations"] - sw["iterations"]) <= 1
    for f in fs:
        assert rel(f["T"], ref["T"]) <= 1e-9
        assert rel(f["T"], fw["T"]) <= 1e-10
        assert rel(f["q"], fw["q"]) <= 1e-8
        assert rel(f["Tband"], fw["Tband"]) <= 1e-10
    # the updates of a sharded solve add up to the whole solve's
    assert sum(s["updates"] for s in ss) == ss[0]["iterations"] * sw["num_cells"] * sw["num_bands"] * \
        sw["num_directions"]


def test_fp32_shards_follow_the_whole_solve():
    d = decks.config2_deck(h_nm=6.0, n_bands=8, n_phi=8, seed=1)
    fw, _ = solve_whole(d, g.GBTE_FP32_MIXED, max_iter=30, err_temp=0.0, err_flux=0.0)
    fs, _, _ = solve_sharded(d, 3, g.GBTE_FP32_MIXED, max_iter=30, err_temp=0.0, err_flux=0.0)
    for f in fs:
        for k in ("T", "q", "Tband"):
            assert rel(f[k], fw[k]) <= 1e-5, (k, rel(f[k], fw[k]))


def test_failed_exchange_is_reported_and_the_handle_stays_usable():
    deck, ref = mg.load("porous_msh")
    hs = [g.StaticBTESynthetic.from_deck(deck, precision=g.GBTE_FP64) for _ in range(2)]
    x = shard.ThreadExchange(2, timeout=60.0)
    count = {"n": 0}
    inner = x.member(1)

    def failing(buf, n, stream):
        count["n"] += 1
        if count["n"] == 5:
            raise RuntimeError("peer lost")
        inner(buf, n, stream)

    blocks = shard.direction_blocks(hs[0].num_directions, 2)
    hs[0].set_direction_shard(*blocks[0], x.member(0))
    hs[1].set_direction_shard(*blocks[1], failing)
    for h in hs:
        h.set_initial(ref["Tf"])
    with pytest.raises(g.GBTEError) as ei:
        shard.solve_sharded(hs, x, max_iter=10, err_temp=0.0, err_flux=0.0)
    assert ei.value.status == g.GBTE_ERR_EXCHANGE
    # back to all directions: the handle solves on its own
    hs[0].set_direction_shard(0, 0, None)
    hs[0].set_initial(ref["Tf"])
    hs[0].solve(allow_not_converged=False)
    assert rel(hs[0].fields()["T"], ref["T"]) <= 1e-9
    for h in hs:
        h.close()


def test_shard_arguments_and_adjoint_are_checked():
    deck, ref = mg.load("porous_msh")
    s = g.StaticBTESynthetic.from_deck(deck, precision=g.GBTE_FP64)
    nd = s.num_directions
    with pytest.raises(g.GBTEError) as ei:
        s.set_direction_shard(nd - 1, 2, lambda b, n, st: None)
    assert ei.value.status == -1
    x = shard.ThreadExchange(1)
    s.set_direction_shard(0, nd, x.member(0))
    s.set_initial(ref["Tf"])
    s.solve(max_iter=3, err_temp=0.0, err_flux=0.0)
    with pytest.raises(g.GBTEError) as ei:
        s.vjp(T_bar=np.ones(s.num_cells), max_iter=2, tol=1e-3)
    assert ei.value.status == -8
    s.close()


def _nccl_child(rank, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    import giftbte_b200 as gg
    import make_golden as mgc
    from giftbte_b200 import shard as sh

    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        deck, ref = mgc.load("porous_msh")
        s = gg.StaticBTESynthetic.from_deck(deck, precision=gg.GBTE_FP64)
        s.set_direction_shard(0, s.num_directions, sh.torch_exchange())
        s.set_initial(ref["Tf"])
        st = s.solve(max_iter=15, err_temp=0.0, err_flux=0.0)
        f = s.fields()
        s.close()
        out["res"] = (st["iterations"], f["T"].tolist(), f["q"].tolist())
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(600)
def test_nccl_exchange_one_rank_is_the_whole_solve():
    # the torch.distributed exchange on the solver's stream, over a
    # one-rank NCCL group (its all-reduce leaves the buffer as it is)
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    with mp.get_context("spawn").Manager() as man:
        out = man.dict()
        mp.start_processes(_nccl_child, args=(port, out), nprocs=1, join=True, start_method="spawn")
        it, T, q = out["res"]
    deck, ref = mg.load("porous_msh")
    fw, _ = solve_whole(deck, g.GBTE_FP64, ref["Tf"], max_iter=15, err_temp=0.0, err_flux=0.0)
    assert it == 15
    assert np.array_equal(np.asarray(T), fw["T"])
    assert np.array_equal(np.asarray(q), fw["q"])
