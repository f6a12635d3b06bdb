"""Sharding of independent search units over ranks (one process per GPU).

Starting states, seeds and graphs are independent units: each rank takes a
contiguous share, runs it with no data-path collective, and only the best
result crosses ranks at the end (its value, the winning rank, and that rank's
bit string). The reference has no multi-device path; this module only splits
the work of its single-device loop (spin_glass_solver.py:586-717) and picks
the best result with a fixed tie rule: the highest value, then the lowest rank.

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
