"""Batched local search: many graphs and many starting states in one launch.

``BatchedSearch`` packs prepared graphs (``DeviceGraph``) into the device
descriptor array of ``pqi_batch_search`` and runs iterated local search for a
list of (graph, starting state) tasks: steepest single-flip ascent, then
forced kicks drawn uniformly or from a learned proposal distribution, repeated
``rounds`` times, best state kept per task. Integer-weight graphs and
float-weight graphs run in separate launches (the gain type differs).
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from . import device as D

_DESC = np.dtype([("W", "<u8"), ("n", "<i4"), ("ld", "<i4"), ("kind", "<i4"), ("pad", "<i4"), ("upper_sum", "<f8")])


class BatchedSearch:
    """Iterated local search over a set of prepared graphs sharing one weight kind."""

    def __init__(self, graphs: list[D.DeviceGraph], stream=None):
        if not graphs:
            raise ValueError("no graphs")
        kinds = {g.w.kind for g in graphs}
        if len(kinds) != 1:
            raise ValueError("graphs of one batch must share the weight kind (int8 or float)")
        assert _lib.load().pqi_batch_graph_desc_bytes() == _DESC.itemsize
        self.graphs = graphs
        self.kind = kinds.pop()
        self.device = graphs[0].device
        self.stream = stream
        self.max_n = max(g.n for g in graphs)
        self.pitch = (self.max_n + 31) // 32
        desc = np.zeros(len(graphs), dtype=_DESC)
        for i, g in enumerate(graphs):
            desc[i]["W"] = g.w.W_i8 if self.kind == _lib.PQI_W_I8 else g.w.W_f32z
            desc[i]["n"] = g.n
            desc[i]["ld"] = g.ld
            desc[i]["kind"] = g.w.kind
            desc[i]["upper_sum"] = g.upper_sum
        self.desc = torch.from_numpy(desc.view(np.uint8).copy()).to(self.device)
        self.n = np.array([g.n for g in graphs], dtype=np.int64)

    def pack_states(self, task_graph, states) -> torch.Tensor:
        """list/array of bool[n_g] per task -> device words [tasks, pitch]."""
        tasks = len(task_graph)
        out = np.zeros((tasks, self.pitch), dtype=np.uint32)
        for t, (g, s) in enumerate(zip(task_graph, states)):
            b = np.asarray(s, dtype=np.bool_)
            n = int(self.n[g])
            pad = np.zeros(self.pitch * 32, dtype=np.bool_)
            pad[:n] = b[:n]
            out[t] = np.packbits(pad.reshape(-1, 8), axis=1, bitorder="little").reshape(-1).view(np.uint32)
        return torch.from_numpy(out.view(np.int32)).to(self.device)

    def random_states(self, task_graph, seed: int) -> torch.Tensor:
        """Uniform random starting states on the device (packed words)."""
        gen = torch.Generator(device=self.device)
        gen.manual_seed(int(seed))
        tasks = len(task_graph)
        w = torch.randint(-(2**31), 2**31 - 1, (tasks, self.pitch), dtype=torch.int64, device=self.device, generator=gen)
        w = w.to(torch.int32)
        # clear bits at and beyond each task's n
        n = torch.from_numpy(self.n[np.asarray(task_graph)]).to(self.device)
        col = torch.arange(self.pitch, device=self.device)[None, :] * 32
        rem = (n[:, None] - col).clamp(0, 32)
        mask = torch.where(rem >= 32, torch.full_like(rem, -1), (torch.ones_like(rem) << rem) - 1)
        return (w & mask.to(torch.int32)).contiguous()

    def run(self, task_graph, init_words: torch.Tensor, is_spin_glass: bool, rounds: int = 0, kick: int = 4,
            seed: int = 0, kick_cdf: torch.Tensor | None = None, cdf_offset: torch.Tensor | None = None,
            flip_budget: int | None = None):
        tg = torch.as_tensor(np.asarray(task_graph, dtype=np.int32)).to(self.device)
        tasks = int(tg.numel())
        best_states = torch.zeros(tasks * self.pitch, dtype=torch.int32, device=self.device)
        best_values = torch.empty(tasks, dtype=torch.float64, device=self.device)
        flips = torch.zeros(1, dtype=torch.int64, device=self.device)
        status = torch.zeros(1, dtype=torch.int32, device=self.device)
        budget = int(flip_budget) if flip_budget is not None else 4 * self.max_n + 64
        _lib.call(
            "pqi_batch_search",
            D._ptr(self.desc),
            len(self.graphs),
            D._ptr(tg),
            D._ptr(init_words),
            self.pitch,
            tasks,
            self.max_n,
            int(self.kind),
            int(bool(is_spin_glass)),
            int(rounds),
            int(kick),
            budget,
            ctypes.c_uint64(int(seed) & 0xFFFFFFFFFFFFFFFF),
            D._ptr(kick_cdf),
            D._ptr(cdf_offset),
            D._ptr(best_states),
            D._ptr(best_values),
            D._ptr(flips),
            D._ptr(status),
            D.stream_ptr(self.stream),
        )
        return best_values, best_states.view(tasks, self.pitch), flips, status

    def cluster_ascent(self, task_graph, init_words: torch.Tensor, is_spin_glass: bool, cluster_size: int = 8,
                       flip_budget: int | None = None):
        """Steepest ascent with one thread-block cluster per task: the same
        result as run(rounds=0), lower latency per flip for large n."""
        tg = torch.as_tensor(np.asarray(task_graph, dtype=np.int32)).to(self.device)
        tasks = int(tg.numel())
        best_states = torch.zeros(tasks * self.pitch, dtype=torch.int32, device=self.device)
        best_values = torch.empty(tasks, dtype=torch.float64, device=self.device)
        flips = torch.zeros(1, dtype=torch.int64, device=self.device)
        status = torch.zeros(1, dtype=torch.int32, device=self.device)
        budget = int(flip_budget) if flip_budget is not None else 4 * self.max_n + 64
        _lib.call(
            "pqi_cluster_ascent",
            D._ptr(self.desc),
            len(self.graphs),
            D._ptr(tg),
            D._ptr(init_words),
            self.pitch,
            tasks,
            self.max_n,
            int(self.kind),
            int(bool(is_spin_glass)),
            int(cluster_size),
            budget,
            D._ptr(best_states),
            D._ptr(best_values),
            D._ptr(flips),
            D._ptr(status),
            D.stream_ptr(self.stream),
        )
        return best_values, best_states.view(tasks, self.pitch), flips, status

    def unpack(self, words: torch.Tensor, task_graph) -> list:
        w = words.cpu().numpy().view(np.uint32)
        out = []
        for t, g in enumerate(task_graph):
            bits = np.unpackbits(w[t].view(np.uint8), bitorder="little")[: int(self.n[g])].astype(np.bool_)
            out.append(bits)
        return out
