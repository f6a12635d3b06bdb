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
from .maxcut_tfim import row_lists as _row_lists  # (kept on each DeviceGraph, alive with it)

_DESC = np.dtype([("W", "<u8"), ("n", "<i4"), ("ld", "<i4"), ("kind", "<i4"), ("pad", "<i4"), ("upper_sum", "<f8"),
                  ("adj_ptr", "<u8"), ("adj_col", "<u8"), ("adj_val", "<u8")])


class BatchedSearch:
    """Iterated local search over a set of prepared graphs sharing one weight kind."""

    def __init__(self, graphs: list[D.DeviceGraph], stream=None, row_lists: bool = True):
        """row_lists: give sparse graphs (at most a quarter of W nonzero) their
        row lists, so the CTA form's starting fields cost O(nonzeros). A float
        graph below 2048 nodes then sums its starting fields in column order
        instead of by warp shuffles: the same values up to float64 rounding, so
        its search may end at a different (still local, float64-exact) optimum
        than with row_lists=False; integer graphs and float graphs of 2048+
        nodes give identical searches either way."""
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
            rl = _row_lists(g) if row_lists else None
            if rl is not None:
                desc[i]["adj_ptr"] = rl[0].data_ptr()
                desc[i]["adj_col"] = rl[1].data_ptr()
                desc[i]["adj_val"] = rl[2].data_ptr()
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
            flip_budget: int | None = None, variant: str = "cta", warps_per_sm: int = 0, out=None,
            fields: str = "auto"):
        """Iterated local search of every task. variant: "cta" (one CTA of 256
        threads per task, any n), "cta128" / "cta64" (CTAs of 128 / 64 threads:
        two / four times the resident tasks, for small graphs) or "warp" (one
        warp per task, max_n <= 1024); all give the same results.

        fields (CTA forms, float graphs): "f64" keeps float64 local fields;
        "f32" keeps float32 local fields (half the shared memory, four resident
        tasks per SM instead of three) that only rank the candidates: the
        starting value is summed in float64, and each flip's float64 gain,
        summed over the flipped row in the same pass, decides its acceptance
        and is what the running value adds, so every accepted flip improves
        the float64 objective and the returned value is float64-exact. The
        ranking can differ from float64 fields' where gains agree to float32
        rounding. "auto" (default): "f64" while its fields fit in shared
        memory (up to 24576 nodes; it is also the faster form there: SK
        n = 8192 flip updates run at 0.50 of HBM bandwidth against 0.35 with
        "f32"), "f32" beyond.
        Integer graphs are exact either way.

        `out` = (best_states, best_values, flips, status) device buffers to
        fill (for CUDA-graph capture); flips and status are accumulated into,
        so zero them between uses."""
        tg = task_graph if torch.is_tensor(task_graph) else torch.as_tensor(np.asarray(task_graph, dtype=np.int32)).to(self.device)
        tasks = int(tg.numel())
        if out is None:
            best_states = torch.zeros(tasks * self.pitch, dtype=torch.int32, device=self.device)
            best_values = torch.empty(tasks, dtype=torch.float64, device=self.device)
            flips = torch.zeros(1, dtype=torch.int64, device=self.device)
            status = torch.zeros(1, dtype=torch.int32, device=self.device)
        else:
            best_states, best_values, flips, status = out
        budget = int(flip_budget) if flip_budget is not None else 4 * self.max_n + 64
        if variant == "warp":
            _lib.call(
                "pqi_batch_search_warp", D._ptr(self.desc), len(self.graphs), D._ptr(tg), D._ptr(init_words),
                self.pitch, tasks, self.max_n, int(self.kind), int(bool(is_spin_glass)), int(rounds), int(kick),
                budget, ctypes.c_uint64(int(seed) & 0xFFFFFFFFFFFFFFFF), D._ptr(kick_cdf), D._ptr(cdf_offset),
                D._ptr(best_states), D._ptr(best_values), D._ptr(flips), D._ptr(status), int(warps_per_sm),
                D.stream_ptr(self.stream),
            )
            return best_values, best_states.view(tasks, self.pitch), flips, status
        if variant not in ("cta", "cta128", "cta64"):
            raise ValueError("variant must be 'cta', 'cta128', 'cta64' or 'warp'")
        if fields == "auto":
            fields = "f32" if self.kind != _lib.PQI_W_I8 and self.max_n > 24576 else "f64"
        if fields not in ("f64", "f32"):
            raise ValueError("fields must be 'f64', 'f32' or 'auto'")
        if variant in ("cta128", "cta64"):
            _lib.call(
                "pqi_batch_search_cta", D._ptr(self.desc), len(self.graphs), D._ptr(tg), D._ptr(init_words),
                self.pitch, tasks, self.max_n, int(self.kind), int(bool(is_spin_glass)), int(rounds), int(kick),
                budget, ctypes.c_uint64(int(seed) & 0xFFFFFFFFFFFFFFFF), D._ptr(kick_cdf), D._ptr(cdf_offset),
                D._ptr(best_states), D._ptr(best_values), D._ptr(flips), D._ptr(status), int(variant[3:]),
                int(fields == "f32"), D.stream_ptr(self.stream),
            )
            return best_values, best_states.view(tasks, self.pitch), flips, status
        _lib.call(
            "pqi_batch_search_f32" if fields == "f32" else "pqi_batch_search",
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
                       flip_budget: int | None = None, target: float | None = None):
        """Steepest ascent with one thread-block cluster per task: the same
        result as run(rounds=0), lower latency per flip for large n.
        target: stop every task soon after the first one whose running value
        reaches it (each task's state and value where it stopped)."""
        tg = torch.as_tensor(np.asarray(task_graph, dtype=np.int32)).to(self.device)
        tasks = int(tg.numel())
        best_states = torch.zeros(tasks * self.pitch, dtype=torch.int32, device=self.device)
        best_values = torch.empty(tasks, dtype=torch.float64, device=self.device)
        flips = torch.zeros(1, dtype=torch.int64, device=self.device)
        status = torch.zeros(1, dtype=torch.int32, device=self.device)
        budget = int(flip_budget) if flip_budget is not None else 4 * self.max_n + 64
        reached = torch.zeros(1, dtype=torch.int32, device=self.device) if target is not None else None
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
            ctypes.c_double(float(target) if target is not None else 0.0),
            D._ptr(reached) if reached is not None else None,
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


class BatchedSolver:
    """Many graphs of mixed weight kinds, many starting states per graph.

    Graphs are grouped by weight kind (int8 vs float32 launches). For each
    group a small autotuner times the kernel forms (one CTA of 256, 128 or 64
    threads per task, or one warp per task with an occupancy cap) on the
    group's tasks and keeps the fastest; `capture()` then records every launch of a step in one CUDA
    graph, so a step is one graph replay. Results are the best value and state
    per graph over its seeds.

    Multi-GPU (``dist``, an initialised torch.distributed module, one process
    per GPU): every rank runs the contiguous share [lo, hi) of each graph's
    seeds (``distributed.shard_range``) with no collective in the search, and
    ``results()`` exchanges once (``distributed.sharded_best``): per graph the
    best value, then the lowest seed. Starting states are drawn for all seeds
    and sliced, so a rank's starts are the ones a single rank would use; with
    rounds = 0 the merged result equals the single-rank result. (With kicks,
    the kick stream depends on the task's position in the rank's launch, and
    ranks above 0 use the seed of ``distributed.shard_seed``.) dist=None is
    the same code path with one rank.
    """

    FORMS = (("cta", 0), ("cta128", 0), ("cta64", 0), ("warp", 0), ("warp", 16), ("warp", 8))

    def __init__(self, graphs: list[D.DeviceGraph], seeds_per_graph: int, is_spin_glass: bool,
                 rounds: int = 0, kick: int = 8, seed: int = 0, stream=None, dist=None):
        from . import distributed as DI

        if seeds_per_graph < 1:
            raise ValueError("seeds_per_graph must be >= 1")
        self.graphs = graphs
        self.S = int(seeds_per_graph)
        self.dist = dist
        world, rank = DI.world_rank(dist)
        if self.S < world:
            raise ValueError("seeds_per_graph must be at least the world size")
        self.lo, self.hi = DI.shard_range(self.S, rank, world)
        self.S_local = self.hi - self.lo
        self.spin = bool(is_spin_glass)
        self.rounds, self.kick = int(rounds), int(kick)
        self.seed = int(seed) if rank == 0 else DI.shard_seed(int(seed), rank)
        self.stream = stream
        self.groups = []
        for kind in sorted({g.w.kind for g in graphs}):
            idx = [i for i, g in enumerate(graphs) if g.w.kind == kind]
            bs = BatchedSearch([graphs[i] for i in idx], stream=stream)
            tg = np.repeat(np.arange(len(idx), dtype=np.int32), self.S_local)
            self.groups.append({
                "kind": kind, "index": idx, "bs": bs,
                "tg": torch.from_numpy(tg).to(bs.device),
                "form": ("cta", 0),
            })
        self.graph = None
        self.tuning = {}

    def autotune(self, sample_tasks: int | None = None, reps: int = 2):
        """Time each kernel form on every group's tasks (or on a sample of
        them, graphs taken evenly across the group) and keep the fastest.
        The full task set is the default: a persistent launch's speed depends
        on how many tasks each resident CTA or warp gets, which a small sample
        does not show."""
        for grp in self.groups:
            bs = grp["bs"]
            tasks = int(grp["tg"].numel())
            count = tasks if sample_tasks is None else min(int(sample_tasks), tasks)
            take = np.linspace(0, tasks - 1, num=count).astype(np.int64)
            tg = grp["tg"][torch.from_numpy(take).to(bs.device)].contiguous()
            words = bs.random_states(tg.cpu().numpy(), seed=self.seed + 99)
            times = {}
            for form, wps in self.FORMS:
                if (form == "warp" and bs.max_n > 1024) or (form in ("cta128", "cta64") and bs.max_n > 2048):
                    continue
                best = float("inf")
                for _ in range(reps + 1):  # first run warms the launch
                    s0 = torch.cuda.Event(enable_timing=True)
                    s1 = torch.cuda.Event(enable_timing=True)
                    s0.record()
                    bs.run(tg, words, self.spin, rounds=self.rounds, kick=self.kick, seed=self.seed,
                           variant=form, warps_per_sm=wps)
                    s1.record()
                    s1.synchronize()
                    best = min(best, s0.elapsed_time(s1))
                times[(form, wps)] = best
            grp["form"] = min(times, key=times.get)
            self.tuning[int(grp["kind"])] = {f"{k[0]}/{k[1]}": v for k, v in times.items()}
        return self.tuning

    def _buffers(self):
        for grp in self.groups:
            bs = grp["bs"]
            tasks = int(grp["tg"].numel())
            grp["init"] = torch.zeros(tasks, bs.pitch, dtype=torch.int32, device=bs.device)
            grp["out"] = (
                torch.zeros(tasks * bs.pitch, dtype=torch.int32, device=bs.device),
                torch.empty(tasks, dtype=torch.float64, device=bs.device),
                torch.zeros(1, dtype=torch.int64, device=bs.device),
                torch.zeros(1, dtype=torch.int32, device=bs.device),
            )

    def set_starts(self, seed: int):
        """Fresh uniform random starting states for every task (device side):
        drawn for all seeds of every graph, this rank's share kept."""
        if "init" not in self.groups[0]:
            self._buffers()
        for grp in self.groups:
            bs = grp["bs"]
            ng = len(grp["index"])
            full = bs.random_states(np.repeat(np.arange(ng, dtype=np.int32), self.S), seed=seed)
            share = full.view(ng, self.S, bs.pitch)[:, self.lo:self.hi].reshape(-1, bs.pitch)
            grp["init"].copy_(share)

    def _launch_all(self):
        for grp in self.groups:
            bs = grp["bs"]
            st, bv, fl, stt = grp["out"]
            fl.zero_()
            stt.zero_()
            form, wps = grp["form"]
            bs.run(grp["tg"], grp["init"], self.spin, rounds=self.rounds, kick=self.kick, seed=self.seed,
                   variant=form, warps_per_sm=wps, out=grp["out"])

    def capture(self):
        """Record one step (every group's launch) in a CUDA graph."""
        if "init" not in self.groups[0]:
            self._buffers()
        self._launch_all()  # warm: function attributes, occupancy queries
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._launch_all()
        self.graph = g
        return g

    def step(self):
        """One step: replay the captured graph (or launch directly)."""
        if self.graph is not None:
            self.graph.replay()
        else:
            self._launch_all()

    def results(self):
        """(best value per graph [G] float64, best state words per graph, flips,
        status), over all ranks when the solver is sharded: the per-seed results
        of this rank's share go through ``distributed.sharded_best`` (one
        exchange of values, one of the winners' words)."""
        from . import distributed as DI

        G = len(self.graphs)
        dev = self.groups[0]["bs"].device
        P = max(grp["bs"].pitch for grp in self.groups)
        vals = np.empty((G, self.S_local), dtype=np.float64)
        words = np.zeros((G, self.S_local, P), dtype=np.uint32)
        flips = 0
        status = 0
        for grp in self.groups:
            bs = grp["bs"]
            st, bv, fl, stt = grp["out"]
            idx = np.asarray(grp["index"])
            vals[idx] = bv.view(-1, self.S_local).cpu().numpy()
            words[idx, :, : bs.pitch] = st.view(-1, self.S_local, bs.pitch).cpu().numpy().view(np.uint32)
            flips += int(fl.item())
            status = max(status, int(stt.item()))
        cdev = DI.collective_device(self.dist)
        best_v, _, best_w = DI.sharded_best(G, self.S, lambda lo, hi: (vals, words), self.dist, cdev)
        world, _ = DI.world_rank(self.dist)
        if world > 1:
            tf = torch.tensor([flips], dtype=torch.int64, device=cdev)
            ts = torch.tensor([status], dtype=torch.int64, device=cdev)
            self.dist.all_reduce(tf, op=self.dist.ReduceOp.SUM)
            self.dist.all_reduce(ts, op=self.dist.ReduceOp.MAX)
            flips, status = int(tf.item()), int(ts.item())
        pitch = {gi: grp["bs"].pitch for grp in self.groups for gi in grp["index"]}
        values = torch.from_numpy(best_v).to(dev)
        states = [torch.from_numpy(best_w[gi, : pitch[gi]].view(np.int32).copy()).to(dev) for gi in range(G)]
        return values, states, flips, status
