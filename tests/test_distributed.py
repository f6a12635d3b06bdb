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


def _solve_graphs():
    from pyqrackising_b200 import workloads as wl

    return [wl.gnp_weighted(40, 0.3, seed=1, dist="normal"), wl.regular_pm1_fast(36, seed=2),
            wl.gnp_weighted(29, 0.5, seed=3, dist="uniform")]


def _host_evaluate(Ws, seeds):
    """The oracle's steepest ascent (the batched kernels' rule) from the
    starting state of each (graph, seed): states depend only on the global
    seed index, as the solver's do. Test infrastructure: the product's
    evaluator is the GPU batch."""
    from oracle import oracle as O

    P = max((W.shape[0] + 31) // 32 for W in Ws)

    def evaluate(lo, hi):
        vals = np.empty((len(Ws), hi - lo))
        words = np.zeros((len(Ws), hi - lo, P), dtype=np.uint32)
        for g, W in enumerate(Ws):
            n = W.shape[0]
            starts = np.random.default_rng(g).random((seeds, n)) < 0.5
            for j, s in enumerate(range(lo, hi)):
                bits, _ = O.steepest_ascent(W, starts[s])
                vals[g, j] = O.compute_energy(bits, W)
                w = O.pack32(bits[None, :])
                words[g, j, : w.size] = w.reshape(-1)
        return vals, words

    return evaluate


def _solve_worker(rank, world, port, seeds, q):
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        import datetime

        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        from pyqrackising_b200.distributed import sharded_best

        Ws = _solve_graphs()
        out = sharded_best(len(Ws), seeds, _host_evaluate(Ws, seeds), dist)
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, out))
    except Exception as ex:  # report to the parent instead of hanging it
        q.put((rank, ex))


@pytest.mark.parametrize("world,seeds", [(2, 5), (3, 7)])
def test_sharded_solve_equals_single_rank(world, seeds):
    """The batched solver's loop (distributed.sharded_best) on gloo ranks, each
    running its share of every graph's seeds: every rank ends with exactly the
    single-rank result (best value, its global seed, its bit string)."""
    from pyqrackising_b200.distributed import sharded_best

    Ws = _solve_graphs()
    ref_v, ref_s, ref_w = sharded_best(len(Ws), seeds, _host_evaluate(Ws, seeds), None)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_solve_worker, args=(r, world, port, seeds, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        rank, out = q.get(timeout=180)
        assert not isinstance(out, Exception), out
        res[rank] = out
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        v, s, w = res[r]
        assert np.array_equal(v, ref_v) and np.array_equal(s, ref_s) and np.array_equal(w, ref_w)


def _spread_worker(rank, world, port, q):
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        import datetime

        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        from pyqrackising_b200.distributed import sharded_best

        out = sharded_best(6, 9, _spread_evaluate, dist)
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, out))
    except Exception as ex:  # report to the parent instead of hanging it
        q.put((rank, ex))


def _spread_evaluate(lo, hi):
    """Unit u's best seed is (2u + 1) mod 9, with a tie at seed 8 for u = 0
    (the lower seed must win), so winners lie in every rank's share."""
    vals = np.zeros((6, hi - lo))
    words = np.zeros((6, hi - lo, 2), dtype=np.uint32)
    for u in range(6):
        for j, s in enumerate(range(lo, hi)):
            vals[u, j] = 10.0 if s == (2 * u + 1) % 9 or (u == 0 and s == 8) else float(s % 3)
            words[u, j] = [u, s]
    return vals, words


def test_sharded_best_spread_winners_and_ties():
    from pyqrackising_b200.distributed import sharded_best

    ref = sharded_best(6, 9, _spread_evaluate, None)
    assert list(ref[1]) == [1, 3, 5, 7, 0, 2]
    world = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_spread_worker, args=(r, world, port, q)) for r in range(world)]
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
    for r in range(world):
        for a, b in zip(res[r], ref):
            assert np.array_equal(a, b)


def test_sharded_solve_rejects_fewer_seeds_than_ranks():
    from pyqrackising_b200.distributed import sharded_best

    class One:
        @staticmethod
        def is_available():
            return True

        @staticmethod
        def is_initialized():
            return True

        @staticmethod
        def get_world_size():
            return 4

        @staticmethod
        def get_rank():
            return 0

    with pytest.raises(ValueError):
        sharded_best(2, 3, lambda lo, hi: None, One)
