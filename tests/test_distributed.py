"""Multi-process sharding logic on CPU (gloo, world size 2): work split, per-rank
seeds, best-over-ranks with its tie rule and the winner's bit string, and the
max-over-ranks timing reduction used by bench.py."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, case, q):
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        import datetime

        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        from pyqrackising_b200.distributed import best_over_ranks, max_over_ranks, shard_range

        out = {}
        lo, hi = shard_range(1001, rank, world)
        out["range"] = (lo, hi)
        words = np.full(5, 100 + rank, dtype=np.uint32)
        if case == "distinct":
            val = [3.5, 7.25][rank]
        elif case == "tie":
            val = 4.0
        else:  # nan on one rank
            val = [float("nan"), -2.0][rank]
        out["best"] = best_over_ranks(val, words, dist)
        out["tmax"] = max_over_ranks([0.5, 1.5][rank], dist)
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, out))
    except Exception as ex:  # report to the parent instead of hanging it
        q.put((rank, ex))


@pytest.mark.parametrize("case,winner,value", [("distinct", 1, 7.25), ("tie", 0, 4.0), ("nan", 1, -2.0)])
def test_best_over_ranks_gloo(case, winner, value):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, case, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        rank, out = q.get(timeout=120)
        assert not isinstance(out, Exception), out
        res[rank] = out
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # contiguous cover of 1001 units
    assert res[0]["range"] == (0, 500) and res[1]["range"] == (500, 1001)
    for r in range(world):
        bv, bw, words = res[r]["best"]
        assert bw == winner and bv == value
        assert np.array_equal(words, np.full(5, 100 + winner, dtype=np.uint32))
        assert res[r]["tmax"] == 1.5


def test_shard_helpers_single_process():
    from pyqrackising_b200.distributed import best_over_ranks, shard_range, shard_seed

    covered = []
    for r in range(7):
        lo, hi = shard_range(50, r, 7)
        covered.extend(range(lo, hi))
    assert covered == list(range(50))
    assert len({shard_seed(3, r) for r in range(8)}) == 8
    v, w, words = best_over_ranks(1.5, np.arange(3, dtype=np.uint32))
    assert (v, w) == (1.5, 0) and np.array_equal(words, np.arange(3, dtype=np.uint32))
    with pytest.raises(ValueError):
        shard_range(10, 3, 3)
