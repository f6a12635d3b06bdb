"""Sharding of independent search units over ranks (one process per GPU).

Starting states, seeds and graphs are independent units: each rank takes a
contiguous share, runs it with no data-path collective, and only the best
result crosses ranks at the end (its value, the winning rank, and that rank's
bit string). The reference has no multi-device path; this module only splits
the work of its single-device loop (spin_glass_solver.py:586-717) and picks
the best result with a fixed tie rule: the highest value, then the lowest rank.

``sharded_best`` is the loop the batched solver runs for one rank or many:
every rank evaluates its contiguous share of the seeds of every graph, keeps
the first best seed per graph, and one exchange (all ranks' values, then the
winners' bit strings) gives every rank the result a single rank would return,
since the ranks' shares are contiguous and in rank order.

Works with any torch.distributed backend: CPU tensors with gloo, CUDA tensors
with nccl (pass device="cuda").
"""

from __future__ import annotations

import numpy as np
import torch


def shard_range(total: int, rank: int, world: int) -> tuple[int, int]:
    """[lo, hi) of `total` units owned by `rank` (contiguous, sizes differ by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    if total < 0:
        raise ValueError("total must be >= 0")
    lo = (total * rank) // world
    hi = (total * (rank + 1)) // world
    return lo, hi


def world_rank(dist=None) -> tuple[int, int]:
    """(world size, rank) of an initialised process group, else (1, 0)."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return 1, 0
    return dist.get_world_size(), dist.get_rank()


def collective_device(dist=None) -> str:
    """Where the exchange tensors live: the current CUDA device for nccl, else the CPU."""
    if dist is not None and dist.is_available() and dist.is_initialized() and dist.get_backend() == "nccl":
        return f"cuda:{torch.cuda.current_device()}"
    return "cpu"


def shard_seed(base_seed: int, rank: int) -> int:
    """Per-rank seed derived from one base seed (ranks draw different starts)."""
    return (int(base_seed) * 1000003 + 7919 * int(rank)) & 0x7FFFFFFF


def best_over_ranks(value: float, words, dist=None, device: str = "cpu"):
    """Pick the best (value, bit string) over all ranks.

    value: this rank's best value (higher is better; NaN counts as lowest).
    words: this rank's bit string as uint32 words (numpy or tensor); every rank
    passes the same number of words.
    Returns (best_value, winner_rank, words of the winner as numpy uint32).
    With dist=None (or an uninitialised process group) this rank is the only one.
    """
    w = np.ascontiguousarray(np.asarray(words.cpu() if torch.is_tensor(words) else words).view(np.uint32))
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return float(value), 0, w.copy()
    world = dist.get_world_size()
    v = float(value)
    if v != v:  # NaN loses
        v = -np.inf
    vals = torch.tensor([v], dtype=torch.float64, device=device)
    gathered = [torch.zeros(1, dtype=torch.float64, device=device) for _ in range(world)]
    dist.all_gather(gathered, vals)
    allv = np.array([float(g.item()) for g in gathered])
    winner = int(np.flatnonzero(allv == allv.max())[0])  # highest value, then lowest rank
    buf = torch.from_numpy(w.view(np.int32).copy()).to(device)
    dist.broadcast(buf, src=winner)
    out = buf.cpu().numpy().view(np.uint32).copy()
    return float(allv[winner]), winner, out


def max_over_ranks(x: float, dist=None, device: str = "cpu") -> float:
    """Max of a float over ranks (timing: the slowest rank's elapsed time)."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def best_per_unit_over_ranks(values, words, dist=None, device: str = "cpu"):
    """Best (value, bit string) of each of U units over all ranks, in one
    exchange of the U values and one of the U winners' words.

    values: float64 [U], this rank's best value per unit (NaN loses).
    words: uint32 [U, P], this rank's bit string per unit.
    Returns (values [U] float64, winner rank [U] int, words [U, P] uint32):
    per unit the highest value, then the lowest rank.
    """
    v = np.asarray(values.cpu() if torch.is_tensor(values) else values, dtype=np.float64).copy()
    w = np.ascontiguousarray(np.asarray(words.cpu() if torch.is_tensor(words) else words).view(np.uint32))
    v[np.isnan(v)] = -np.inf
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return v, np.zeros(len(v), dtype=np.int64), w.copy()
    world, rank = dist.get_world_size(), dist.get_rank()
    vt = torch.from_numpy(v).to(device)
    allv = [torch.empty_like(vt) for _ in range(world)]
    dist.all_gather(allv, vt)
    allv = np.stack([a.cpu().numpy() for a in allv])  # [world, U]
    winner = np.argmax(allv, axis=0)  # first maximum: the lowest rank
    # each unit's words from its winner: a sum in which only the winner adds
    mine = np.where((winner == rank)[:, None], w, 0).astype(np.uint32)
    buf = torch.from_numpy(mine.view(np.int32).astype(np.int64)).to(device)
    dist.all_reduce(buf, op=dist.ReduceOp.SUM)
    out = buf.cpu().numpy().astype(np.int64).astype(np.int32).view(np.uint32).reshape(w.shape)
    return allv[winner, np.arange(allv.shape[1])], winner.astype(np.int64), out


def sharded_best(units: int, seeds: int, evaluate, dist=None, device: str = "cpu"):
    """The sharded solve loop: seeds of every unit split over ranks.

    evaluate(lo, hi) runs seeds [lo, hi) of every unit on this rank's device and
    returns (values [units, hi - lo], words [units, hi - lo, P]); a rank with an
    empty share is not called. Per unit the first best seed of the share is
    kept, then ``best_per_unit_over_ranks`` picks over ranks. With dist=None
    this is the single-rank loop.
    Returns (values [units], global seed index [units], words [units, P]).
    """
    world, rank = world_rank(dist)
    if seeds < world:  # the same test on every rank: all raise together
        raise ValueError("every rank needs at least one seed per unit (seeds >= world size)")
    lo, hi = shard_range(seeds, rank, world)
    vals, words = evaluate(lo, hi)
    vals = np.asarray(vals.cpu() if torch.is_tensor(vals) else vals, dtype=np.float64).reshape(units, hi - lo)
    words = np.asarray(words.cpu() if torch.is_tensor(words) else words).view(np.uint32).reshape(units, hi - lo, -1)
    vals = np.where(np.isnan(vals), -np.inf, vals)
    arg = np.argmax(vals, axis=1)  # first maximum: the lowest seed
    best_v = vals[np.arange(units), arg]
    best_w = words[np.arange(units), arg]
    best_s = lo + arg
    if world == 1:
        return best_v, best_s.astype(np.int64), np.ascontiguousarray(best_w)
    v, win, w = best_per_unit_over_ranks(best_v, best_w, dist, device)
    # the winning seed index travels with its rank's words: exchange it too
    seed_idx = np.where(win == rank, best_s, 0).astype(np.int64)
    st = torch.from_numpy(seed_idx).to(device)
    dist.all_reduce(st, op=dist.ReduceOp.SUM)
    return v, st.cpu().numpy().astype(np.int64), w
