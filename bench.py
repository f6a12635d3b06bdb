"""Benchmark of the batched cut-scoring hot path (one JSON line on rank 0).

Workload: dense unweighted MAXCUT, Erdos-Renyi G(n=2048, p=0.5), unit weights,
dense symmetric float32 couplings with a zero diagonal (seeded synthetic, the
shape of the named configuration); one batch = 65536 candidate bit strings
(seeded uniform bits), the batch the reference's maxcut_tfim scores per round
at its default quality 6 for n = 2048 (shots = n << 6, halved and rounded to
32: maxcut_tfim.py:379, :159), scored as calculate_cut does (kernels.cl:44-94)
and selected with its tie rule. One step = one batch.

* value: candidates scored per second over all ranks (cut evals/s), device time
  of the timed steps (CUDA events), inputs already in HBM. L2 is flushed
  (a 256 MB write) between timed steps, outside the timed windows.
* e2e: the same metric through the public path with host buffers: each step
  copies the packed batch from pinned host memory (on a copy stream, double
  buffered so the next step's copy overlaps this step's scoring), scores it
  through the C ABI and reads the (best value, index) pair back.
* roofline: the scoring GEMM (2*B*n^2 integer ops per launch) against the
  int8 tensor rate, taken as twice the measured dense bf16 rate.
* cpu_baseline: the reference's CPU scoring path (numba: compute_cut_diff_between
  per candidate under prange, maxcut_tfim.py:77-136), restated in
  oracle/numba_port.py and pinned to the reference's own values, on all host
  threads over a bounded sample of the batch; beside it the reference's
  OpenCL calculate_cut compiled for the host (oracle/_ref).
* --impl reference: the same CPU scoring as the reference arm, same config.
* time_to_best: the other half of the metric, on the Sherrington-Kirkpatrick
  spin glass (n = 8192, J ~ N(0,1)/sqrt(n) float32): wall time of the plain
  GPU form (spin_glass_solver's local-search loop from one start) against the
  batched form (32 starts, one thread-block cluster each, one launch) until
  each returns; the batched form must reach the plain form's best energy.
  Both values are re-scored in float64 and their relative error reported.

Multi-GPU: every rank scores its own batches (weak scaling); the only
exchange is the max over ranks of the elapsed time.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

N_NODES = 2048
BATCH = 65536
EDGE_P = 0.5
METRIC = "cut evals/s"
UNIT = "candidates/s"


def workload_config(extra=None):
    cfg = {
        "workload": "ER G(n=2048,p=0.5) unit weights, 65536 candidates per batch (maxcut_tfim quality-6 batch), calculate_cut + reference-order argmax",
        "n": N_NODES,
        "batch": BATCH,
        "weights": "int8 (exact)",
        "l2": "flushed between timed device steps (256 MB write); e2e steps take a fresh batch from the host each step",
        "e2e_pipeline": "pinned H2D of each step's packed batch on a copy stream into two alternating device buffers (step i+1's copy overlaps step i's scoring), D2H of (value, index) every step",
    }
    if extra:
        cfg.update(extra)
    return cfg


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), float(p["bf16_tflops"]), "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks sampled every 200 ms while the timed region runs."""

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._proc = None

    def wait_first(self, timeout=3.0):
        """Block until the first sample arrives (so the timed region is covered)."""
        t0 = time.perf_counter()
        while not self.samples and time.perf_counter() - t0 < timeout:
            time.sleep(0.02)

    def __enter__(self):
        try:
            self._proc = subprocess.Popen(
                [
                    "nvidia-smi",
                    f"--id={self.index}",
                    "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
                    "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                    "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                    "--format=csv,noheader,nounits",
                    "-lms",
                    "200",
                ],
                stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL,
                text=True,
            )
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self._proc = None
        return self

    def _read(self):
        for line in self._proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()

    def summary(self):
        sm = [float(s[0]) for s in self.samples if len(s) >= 7 and s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if len(s) >= 7 and s[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            if len(s) >= 7:
                for nm, v in zip(names, s[3:7]):
                    if v.lower() == "active":
                        reasons.add(nm)
        return {
            "sm_mhz": float(np.median(sm)) if sm else None,
            "sm_max_mhz": max(mx) if mx else None,
            "reasons": sorted(reasons),
            "samples": len(self.samples),
        }


def _emulator_or_c_port():
    """The reference's own kernels.cl built for the host (oracle/_ref) when it was
    built in this checkout, else the oracle's C port of it."""
    from oracle import oracle as O

    O.build_oracle()
    return O, ("reference" if O.ref_available() else "port")


def _kernels_cl_sample(O, kind, W, th, sample):
    G, L = O.cut_geometry(sample, 148)
    if kind == "reference":
        # calculate_cut as the reference launches it: G work-items in groups of L
        # host threads, each work-item scoring its grid-stride share
        e, i, _, _ = O.ref_cut_select(W, th, sample, 0, G, L)
    else:
        e, i = O.cut_select(W, th, sample, 0, G, L)
    return e, i


class NumbaScoring:
    """The reference's CPU candidate scoring (numba, maxcut_tfim.py:77-136 with
    compute_cut_diff_between, maxcut_tfim_util.py:445-461) as the oracle restates
    it (oracle/numba_port.py), on all the host threads numba uses; the C port of
    calculate_cut (OpenMP) when numba is absent."""

    def __init__(self, W):
        from oracle import numba_port as P

        self.W = W
        self.numba = P.available()
        if self.numba:
            P.warm()
            self.P = P
            self.cores = P.threads()
            self.kind_text = ("the reference's CPU scoring (numba prange over candidates, compute_cut_diff_between "
                              "against the all-false start, first max) restated in oracle/numba_port.py")
        else:
            from oracle import oracle as O

            O.build_oracle()
            self.O = O
            self.cores = os.cpu_count() or 1
            self.kind_text = "the oracle's C port of calculate_cut (OpenMP over candidates); numba is not installed"

    def __call__(self, X):
        if self.numba:
            return self.P.select_first_max(self.P.score_batch(X, self.W))
        v = self.O.cut_values(self.W, self.O.pack32(X), X.shape[0], 0)
        i = int(np.argmax(v))
        return float(v[i]), i


def cpu_baseline(W, X, sample=2048):
    """The reference's CPU scoring on the host cores over a bounded sample of the
    batch (about 10-20 s of CPU time), plus the reference's kernels.cl run on the
    host (its OpenCL kernel, work-groups concurrent) as a second figure."""
    score = NumbaScoring(W)
    score(X[:64])
    t0 = time.perf_counter()
    score(X[:sample])
    dt = time.perf_counter() - t0
    out = {
        "value": sample / dt,
        "unit": UNIT,
        "cores": score.cores,
        "kind": "port",
        "sample": f"{sample} of the batch's candidates (n={W.shape[0]}) in one call: {score.kind_text}",
    }
    try:
        O, kind = _emulator_or_c_port()
        th = O.pack32(X[:256])
        _kernels_cl_sample(O, kind, W, th[:32], 32)
        t0 = time.perf_counter()
        _kernels_cl_sample(O, kind, W, th, 256)
        dt = time.perf_counter() - t0
        out["kernels_cl_on_host"] = {
            "value": 256 / dt,
            "unit": UNIT,
            "kind": kind,
            "sample": "256 candidates: the reference's calculate_cut (kernels.cl:44-94) compiled for the host, "
                      "160 work-items in groups of 32 threads, all groups at once" if kind == "reference" else
                      "256 candidates: the oracle's C port of calculate_cut",
        }
    except Exception as ex:  # pragma: no cover
        out["kernels_cl_on_host"] = {"unavailable": str(ex)}
    return out


def run_reference(args, rank, world):
    """The reference arm: the reference's CPU scoring of this workload (restated
    in the oracle, see NumbaScoring) on all host threads; each step scores a
    bounded sample of the step's batch. Rank 0 alone runs it."""
    if rank != 0:
        return 0
    W = make_graph()
    sample = 2048
    X = make_batch(0, sample)
    score = NumbaScoring(W)
    for _ in range(max(1, args.warmup)):
        score(X[:128])
    t_steps = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        score(X)
        t_steps.append(time.perf_counter() - t0)
    ms = 1000.0 * float(np.mean(t_steps))
    value = sample / (ms / 1000.0)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": workload_config(),
        "cpu_baseline": {
            "value": value,
            "unit": UNIT,
            "cores": score.cores,
            "kind": "port",
            "sample": f"{sample} of the {BATCH} candidates of a batch per step (the rate is per candidate): {score.kind_text}",
        },
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def time_to_best(n=8192, starts=32, cluster=8):
    """Wall time to the plain GPU form's best energy on SK n=8192 (see module
    doc); each form's median over three runs."""
    import importlib

    import torch

    from pyqrackising_b200 import workloads as wl
    from pyqrackising_b200.batch import BatchedSearch
    from pyqrackising_b200.device import DeviceGraph

    SG = importlib.import_module("pyqrackising_b200.spin_glass_solver")
    W = wl.sherrington_kirkpatrick(n, seed=1)
    dg = DeviceGraph(W)
    start = np.random.default_rng(0).random(n) < 0.5
    bs = BatchedSearch([dg])
    tasks = [0] * starts
    w0 = bs.random_states(tasks, seed=7)
    # one untimed run of each form on this graph (module load, workspaces,
    # first-launch attributes), then the timed runs
    SG.local_search(dg, start, True, n * n, 148, 148, 0.0)
    bs.cluster_ascent(tasks, w0, True, cluster_size=cluster)
    bs.cluster_ascent(tasks, w0, True, cluster_size=cluster, target=0.0)
    torch.cuda.synchronize()

    # each form timed three times (host clock after a device sync), the
    # median reported; every run does the same work
    reps = 3
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        words, _ = SG.local_search(dg, start, True, n * n, 148, 148, 0.0)
        _, e_plain = dg.rescore(words)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    t_plain = float(np.median(times))
    e_plain = float(e_plain.item())

    # the full ascent of every start
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        vals, best, flips, status = bs.cluster_ascent(tasks, w0, True, cluster_size=cluster)
        t_best = int(torch.argmax(vals).item())
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    t_batched = float(np.median(times))
    e_batched = float(vals[t_best].item())
    _, e64 = dg.rescore(best[t_best].contiguous())
    e64 = float(e64.item())
    # the same launch in target mode: every start stops once one reaches the
    # plain form's best (checked every 16 flips on the device)
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        vt, bt, _, st_t = bs.cluster_ascent(tasks, w0, True, cluster_size=cluster, target=e_plain)
        tb = int(torch.argmax(vt).item())
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    t_target = float(np.median(times))
    _, et64 = dg.rescore(bt[tb].contiguous())
    et64 = float(et64.item())
    reached_t = et64 >= e_plain * (1.0 - 1e-5)
    return {
        "workload": f"SK n={n}, J~N(0,1)/sqrt(n) float32, is_spin_glass; plain: local-search loop from 1 start; batched: {starts} starts, cluster ascent ({cluster} CTAs per start)",
        "plain_s": t_plain,
        "plain_energy": e_plain,
        "batched_s": t_batched,
        "batched_energy": e_batched,
        "batched_energy_rel_err_vs_fp64": abs(e_batched - e64) / max(abs(e64), 1e-300),
        "batched_flips": int(flips.item()),
        "batched_status": int(status.item()),
        "reaches_plain_best": e64 >= e_plain * (1.0 - 1e-5),
        "speedup_full_run": t_plain / t_batched,
        "to_target_s": t_target,
        "to_target_energy_fp64": et64,
        "to_target_status": int(st_t.item()),
        "to_target_reaches_plain_best": reached_t,
        "speedup": t_plain / (t_target if reached_t else t_batched),
        "speedup_basis": "plain_s / to_target_s (time until a start holds the plain best)" if reached_t
        else "plain_s / batched_s (target run did not reach)",
    }


def time_to_best_learned(n=8192, starts=32, cluster=8, rounds=4, kick=64, temperature=3.0):
    """The batched + learned form on SK n=8192 against the plain GPU form's
    best energy. Stages, each timed on the host clock after a device sync:
      1. cluster ascent from `starts` random states (one launch);
      2. the network's proposals on each task's optimum (forward per task,
         kick distributions by pqi_mpnn_kick_cdf);
      3. `rounds` of the batched iterated search from those optima with
         learned kicks.
    time_to_plain_best is the first stage run again in target mode (every
    start stops once one holds the plain form's best; a device flag), or else
    the end of the first stage whose running best reaches it (None if none
    does). Beside
    stage 3, the same search with uniform kicks from the same optima, seeds
    and budget: what the network adds over the method without it."""
    import importlib

    import torch

    from pyqrackising_b200 import learned as L
    from pyqrackising_b200 import workloads as wl
    from pyqrackising_b200.batch import BatchedSearch
    from pyqrackising_b200.device import DeviceGraph

    SG = importlib.import_module("pyqrackising_b200.spin_glass_solver")
    W = wl.sherrington_kirkpatrick(n, seed=1)
    dg = DeviceGraph(W)
    net = L.ProposalNet.load(os.path.join(REPO, "pyqrackising_b200", "weights", "proposal_net.pt"))
    start = np.random.default_rng(0).random(n) < 0.5
    bs = BatchedSearch([dg])
    bsT = BatchedSearch([dg] * starts)  # one descriptor (and proposal) per task
    tasks = [0] * starts
    w0 = bs.random_states(tasks, seed=7)
    # untimed warm run of every stage (module load, workspaces, attributes)
    SG.local_search(dg, start, True, n * n, 148, 148, 0.0)
    vA, wA, _, _ = bs.cluster_ascent(tasks, w0, True, cluster_size=cluster)
    cdf, off = L.task_proposals(net, dg, wA, temperature=temperature)
    bsT.run(list(range(starts)), wA.reshape(-1).contiguous(), True, rounds=1, kick=kick, seed=1,
            kick_cdf=cdf, cdf_offset=off)
    torch.cuda.synchronize()

    t0 = time.perf_counter()
    words, _ = SG.local_search(dg, start, True, n * n, 148, 148, 0.0)
    _, e_plain = dg.rescore(words)
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    e_plain = float(e_plain.item())

    def reached(v):
        return v >= e_plain * (1.0 - 1e-5) if e_plain >= 0 else v >= e_plain * (1.0 + 1e-5)

    t0 = time.perf_counter()
    vA, wA, _, _ = bs.cluster_ascent(tasks, w0, True, cluster_size=cluster)
    b1 = float(vA.max().item())
    t1 = time.perf_counter() - t0
    cdf, off = L.task_proposals(net, dg, wA, temperature=temperature)
    torch.cuda.synchronize()
    t2 = time.perf_counter() - t0
    A = wA.reshape(-1).contiguous()
    vP, wP, _, sP = bsT.run(list(range(starts)), A, True, rounds=rounds, kick=kick, seed=3, kick_cdf=cdf,
                            cdf_offset=off)
    b3 = float(vP.max().item())
    t3 = time.perf_counter() - t0
    ta = time.perf_counter()
    vU, _, _, _ = bs.run(tasks, A, True, rounds=rounds, kick=kick, seed=3)
    bU = float(vU.max().item())
    t_uniform = time.perf_counter() - ta
    best = int(torch.argmax(vP).item())
    _, e64 = dg.rescore(wP[best].contiguous())
    # the first stage in target mode: every start stops once one holds the
    # plain form's best (the later stages start from full ascents above)
    bs.cluster_ascent(tasks, w0, True, cluster_size=cluster, target=e_plain)  # warm
    torch.cuda.synchronize()
    tt = time.perf_counter()
    vT, wT, _, _ = bs.cluster_ascent(tasks, w0, True, cluster_size=cluster, target=e_plain)
    bT = float(vT.max().item())
    t_target = time.perf_counter() - tt
    ttb = t_target if reached(bT) else (t1 if reached(b1) else (t3 if reached(max(b1, b3)) else None))
    return {
        "workload": f"SK n={n}, J~N(0,1)/sqrt(n) float32, is_spin_glass; plain: local-search loop from 1 start; "
                    f"batched + learned: {starts} starts, cluster ascent ({cluster} CTAs per start), the trained "
                    f"network's per-task proposals (T={temperature}), {rounds} rounds of batched iterated search "
                    f"with {kick} learned kicks per round",
        "plain_s": t_plain,
        "plain_energy": e_plain,
        "stage_ascent_s": t1, "stage_ascent_best": b1,
        "stage_proposals_s": t2 - t1,
        "stage_learned_search_s": t3 - t2, "stage_learned_search_best": b3,
        "uniform_search_best": bU, "uniform_search_s": t_uniform,
        "learned_minus_uniform": b3 - bU,
        "best_energy_rel_err_vs_fp64": abs(b3 - float(e64.item())) / max(abs(float(e64.item())), 1e-300),
        "status": int(sP.item()),
        "stage_ascent_to_target_s": t_target, "stage_ascent_to_target_best": bT,
        "time_to_plain_best_s": ttb,
        "time_to_plain_best_basis": "the first stage in target mode (the learned stages come after the plain best is reached)",
        "speedup": (t_plain / ttb) if ttb else None,
    }


def scoring_batch_leg(dg, batch=4096, reps=50):
    """The scoring kernel at the parallel seed count of the ER-2048 solve (4096
    candidates, a GEMM 16x smaller than the headline's): device time per call
    (CUDA events around the GEMM launch and around the whole call), the
    fraction of the int8 peak, L2 flushed before each call."""
    import torch

    from oracle import oracle as O
    from pyqrackising_b200 import _lib

    X = np.random.default_rng(77).random((batch, N_NODES)) < 0.5
    words = dg.pack(X)
    G, L = O.cut_geometry(batch, 148)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dg.device)
    for _ in range(5):
        dg.calculate_cut(words, batch, False, G, L, energies=False)
    k_ms, s_ms = [], []
    lib = _lib.load()
    for i in range(reps):
        flush.fill_(i & 0xFF)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ka, kb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        ka.record()
        kb.record()
        lib.pqi_score_set_events(ctypes.c_void_p(ka.cuda_event), ctypes.c_void_p(kb.cuda_event))
        dg.calculate_cut(words, batch, False, G, L, energies=False)
        b.record()
        b.synchronize()
        k_ms.append(ka.elapsed_time(kb))
        s_ms.append(a.elapsed_time(b))
    lib.pqi_score_set_events(None, None)
    _, bf16, src = peaks()
    km = float(np.median(k_ms))
    ops = 2.0 * batch * N_NODES * N_NODES
    return {
        "workload": f"ER G(n=2048,p=0.5) unit weights, {batch} candidates per call (the solve's parallel seeds)",
        "kernel_ms": km,
        "call_ms": float(np.median(s_ms)),
        "candidates_per_s": batch / (float(np.median(s_ms)) / 1e3),
        "frac_of_int8_peak": ops / (km / 1e3) / 1e12 / (2.0 * bf16),
        "peak_basis": f"int8 dense = 2 x bf16 dense ({src} bf16 {bf16} TFLOP/s)",
    }


def e2e_pipeline(dg, batches_host, like, G, L, steps, warmup):
    """Device time (ms) of `steps` end-to-end steps: H2D copy of the step's
    packed batch from pinned memory, scoring through the public call, D2H of
    the selected (value, index). Copies run on their own stream into two
    alternating device buffers."""
    import torch

    nb = len(batches_host)
    pinned = [torch.from_numpy(b.view(np.int32).reshape(-1)).pin_memory() for b in batches_host]
    dev_in = [torch.empty_like(like) for _ in range(2)]
    out_e = torch.empty(steps + warmup, dtype=torch.float32).pin_memory()
    out_i = torch.empty(steps + warmup, dtype=torch.int32).pin_memory()
    comp = torch.cuda.current_stream()
    copy = torch.cuda.Stream()
    copied = [torch.cuda.Event() for _ in range(2)]
    used = [torch.cuda.Event() for _ in range(2)]

    def run(i0, count):
        for i in range(i0, i0 + count):
            buf = i & 1
            with torch.cuda.stream(copy):
                if i >= 2:
                    copy.wait_event(used[buf])  # step i-2 has finished reading this buffer
                dev_in[buf].copy_(pinned[i % nb], non_blocking=True)
                copied[buf].record(copy)
            comp.wait_event(copied[buf])
            _, be, bi = dg.calculate_cut(dev_in[buf], BATCH, False, G, L, energies=False)
            used[buf].record(comp)
            out_e[i].copy_(be[0], non_blocking=True)
            out_i[i].copy_(bi[0], non_blocking=True)

    run(0, warmup)
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(comp)
    copy.wait_stream(comp)
    run(warmup, steps)
    end.record(comp)
    end.synchronize()
    ms = start.elapsed_time(end)
    # the host link alone: the same copies back to back (the pipeline's floor)
    start.record(copy)
    with torch.cuda.stream(copy):
        for i in range(steps):
            dev_in[i & 1].copy_(pinned[i % nb], non_blocking=True)
    end.record(copy)
    end.synchronize()
    e2e_pipeline.h2d_only_ms = start.elapsed_time(end)
    return ms


def plain_small_leg(reps=5):
    """Config 1: spin_glass_solver(W, quality=6, is_spin_glass=True) on the
    3-regular n=64 +-1 fixture from its recorded best_guess, through the public
    call; next to it the reference's GPU-branch driver loop run on the host
    cores with the reference's kernels compiled for the host (or the C port)."""
    import importlib

    import torch

    from oracle import oracle as O

    SG = importlib.import_module("pyqrackising_b200.spin_glass_solver")
    z = np.load(os.path.join(REPO, "tests", "golden", "golden_c1_regular64.npz"))
    W = z["W"]
    guess = [bool(b) for b in z["best_guess"]]
    iters = int(z["e2e_gray_iterations"])
    SG.spin_glass_solver(W, quality=6, is_spin_glass=True, best_guess=guess, gray_iterations=iters)  # warm
    ts = []
    res = None
    for _ in range(reps):
        torch.cuda.synchronize()
        t = time.perf_counter()
        res = SG.spin_glass_solver(W, quality=6, is_spin_glass=True, best_guess=guess, gray_iterations=iters)
        torch.cuda.synchronize()
        ts.append(time.perf_counter() - t)
    use_ref = O.ref_available()
    tc = []
    theta_ref = None
    for _ in range(reps):
        t = time.perf_counter()
        theta_ref = O.spin_glass_gpu_path(W, np.array(guess), True, iters, 148, 148, use_ref=use_ref)[0]
        tc.append(time.perf_counter() - t)
    e_ref = O.compute_energy(theta_ref, W)
    return {
        "workload": "3-regular n=64 +-1 (fixture), spin_glass_solver(quality=6, is_spin_glass=True) from the recorded best_guess",
        "ms": 1e3 * float(np.median(ts)),
        "energy": -float(res[3]),
        "cpu_ms": 1e3 * float(np.median(tc)),
        "cpu_kind": "reference" if use_ref else "port",
        "cpu_energy": float(e_ref),
        "not_below_reference": -float(res[3]) >= float(e_ref) - 1e-9,
    }


def learned_leg():
    """Config 5: the committed trained proposal network on G(16384, 0.01) with
    N(0, 1) weights: the batched iterated search with uniform kicks and with
    the network's per-task proposals from the same optima, each refined by the
    plain local search (the arbiter), next to the plain search alone."""
    from pyqrackising_b200 import learned as L
    from pyqrackising_b200.train_proposals import evaluate

    net = L.ProposalNet.load(os.path.join(REPO, "pyqrackising_b200", "weights", "proposal_net.pt"))
    r = evaluate(net)
    r["weights"] = "pyqrackising_b200/weights/proposal_net.pt (trained on 10,000 streamed graphs)"
    return r


def batched_leg(graphs=512, seeds=256):
    """Batched uneven instances: 512 graphs, n ~ U[64, 1024] (half 3-regular
    +-1 as int8, half G(n, 0.1) with uniform (0, 1] float32 weights), 256
    starting states each; kernel forms autotuned per weight kind; one step
    (steepest ascent of every task) replayed from a captured CUDA graph."""
    import torch

    from pyqrackising_b200 import workloads as wl
    from pyqrackising_b200.batch import BatchedSolver
    from pyqrackising_b200.device import DeviceGraph

    Ws = wl.batched_uneven(graphs, seed=7)
    dgs = [DeviceGraph(W) for W in Ws]
    sol = BatchedSolver(dgs, seeds, True, rounds=0, seed=3)
    tuning = sol.autotune()
    sol.set_starts(11)
    sol.capture()
    for _ in range(2):
        sol.step()
    torch.cuda.synchronize()
    ts = []
    for _ in range(5):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        sol.step()
        b.record()
        b.synchronize()
        ts.append(a.elapsed_time(b))
    values, _, flips, status = sol.results()
    ms = float(np.median(ts))
    tasks = graphs * seeds
    return {
        "workload": f"{graphs} graphs n~U[64,1024] (half 3-regular +-1 int8, half G(n,0.1) U(0,1] float32) x {seeds} starts, steepest ascent per task, one captured CUDA graph per step",
        "ms_per_step": ms,
        "tasks_per_s": tasks / (ms / 1e3),
        "flips_per_step": flips,
        "flips_per_s": flips / (ms / 1e3),
        "forms": {str(g["kind"]): f"{g['form'][0]}/{g['form'][1]}" for g in sol.groups},
        "autotune_ms": tuning,
        "status": status,
        "mean_best_energy": float(values.mean()),
    }


def flip_bandwidth_leg(n=8192, tasks=1776, fields="auto"):
    """Flip updates on the SK spin glass (W = 256 MB float32, larger than L2):
    many starts of the batched ascent at once; each accepted flip reads one W
    row (n * 4 bytes) and updates the task's n local fields. The starting
    fields (O(n^2) per start) are timed in a run with a one-flip budget and
    subtracted; 2048 flips per start keep the flip phase the larger part."""
    import torch

    from pyqrackising_b200 import workloads as wl
    from pyqrackising_b200.batch import BatchedSearch
    from pyqrackising_b200.device import DeviceGraph

    dg = DeviceGraph(wl.sherrington_kirkpatrick(n, seed=1))
    bs = BatchedSearch([dg])
    tg = torch.zeros(tasks, dtype=torch.int32, device=dg.device)
    w0 = bs.random_states(np.zeros(tasks, dtype=np.int32), seed=5)
    bs.run(tg, w0, True, rounds=0, flip_budget=64, fields=fields)  # warm
    torch.cuda.synchronize()
    # starting fields cost n rows per task: time them alone (zero-flip budget
    # is not allowed, so a one-flip budget) and subtract
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    _, _, f1, _ = bs.run(tg, w0, True, rounds=0, flip_budget=1, fields=fields)
    b.record()
    b.synchronize()
    t_init = a.elapsed_time(b)
    a.record()
    v2, b2, f2, st = bs.run(tg, w0, True, rounds=0, flip_budget=1 + 2048, fields=fields)
    b.record()
    b.synchronize()
    t_all = a.elapsed_time(b)
    flips = int(f2.item()) - int(f1.item())
    dt = (t_all - t_init) / 1e3
    hbm, _, src = peaks()
    gbs = flips * n * 4 / dt / 1e9
    # the tracked values against float64 re-scoring of the returned states
    pick = list(range(0, tasks, max(1, tasks // 16)))
    _, e64 = dg.rescore(b2[pick].contiguous(), rows=len(pick))
    tracked = v2[pick]
    rel = float(((tracked - e64).abs() / e64.abs().clamp_min(1e-300)).max().item())
    used = fields if fields != "auto" else ("f32" if n > 24576 else "f64")
    return {
        "workload": f"SK n={n} float32, {tasks} starts of the batched ascent, 2048 flips each after the starting fields (timed apart and subtracted), {used} local fields, float64 acceptance and running value",
        "tracked_value_rel_err_vs_fp64": rel,
        "flips": flips,
        "flips_per_s": flips / dt,
        "row_bytes_per_flip": n * 4,
        "achieved_GBps": gbs,
        "peak_GBps": hbm,
        "frac": gbs / hbm,
        "peak_basis": f"{src} HBM copy bandwidth",
    }


# ----------------------------------------------------------------------------
# Legs outside the headline line: `python bench.py --leg NAME [NAME ...]` runs
# the named legs alone and prints one JSON line per measurement (device time
# by CUDA events on the launching stream; L2 flushed where W exceeds it).
#
#   double   one double-bit-flip pass (kernels.cl:150-231 semantics, from
#            maintained gains) on SK n=8192 float32 and ER(2048, 0.5) int8
#   gray     one Gray-code search (kernels.cl:877-978 semantics) from a
#            single-flip local optimum: SK n=8192 (n^2 iterations, 148 seeds)
#            and ER(1024, 0.5) (n^2/16 iterations)
#   tfim     the TFIM sampler alone (3-regular and ER n=2048, quality 6:
#            65,536 shots) and maxcut_tfim end to end on ER(1024, 0.5), q=2
#   sparse   spin_glass_solver_sparse on G(16384, 0.01) N(0,1) next to the
#            dense solver on the same matrix
#   bnb      solve_maxcut_bnb on 3-regular +-1 graphs, n = 28 and 32
#   flips    a short batched ascent on SK n=8192 (444 starts, 64 flips each,
#            float64 fields; a small case for profiling the flip phase)
#   cluster  a cluster ascent on SK n=8192 (8 starts, 8-CTA clusters), checked
#            against the CTA-per-task form
#   mpnn     one proposal-network forward and backward on G(16384, 0.01)
#   csr      G(200000, 1e-4) N(0,1) on compressed rows: the sparse solver, the
#            double pass and one descent
# A leg exits non-zero when its result disagrees with its check.

_flush_buf = None


def _flush_l2():
    """Write 256 MB (twice the L2) so the next launch starts cold."""
    import torch

    global _flush_buf
    if _flush_buf is None:
        _flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    _flush_buf.fill_(1)


def _timed(fn, reps, flush=True):
    """Mean device time (ms) of fn() over reps launches."""
    import torch

    total = 0.0
    for _ in range(reps):
        if flush:
            _flush_l2()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        total += a.elapsed_time(b)
    return total / reps


def _emit(**kw):
    print(json.dumps(kw), flush=True)


def _local_optimum(dg, seed, spin=True):
    """Random state taken to a single-flip local optimum with the device descent.
    The words hold ceil(n/32) + 1 int32, so they also read as ceil(n/64) 64-bit words."""
    from pyqrackising_b200 import device as D
    from pyqrackising_b200 import workloads as wl

    words = dg.pack(wl.random_bits(dg.n, seed))
    _, g64 = dg.gains(words)
    Gf, Lf = D.geometry(min(D.WORK_GROUP_MULTIPLE, dg.n), dg.n, D.max_gpu_proc_elem())
    while True:
        _, _, rc = dg.single_descent(words, g64, spin, Gf, Lf, 1 << 16)
        if rc != 3:
            break
    return words, g64, Gf, Lf


def leg_double():
    from pyqrackising_b200 import device as D
    from pyqrackising_b200 import workloads as wl

    hbm, _, src = peaks()
    for name, W, spin in (("SK n=8192 float32", wl.sherrington_kirkpatrick(8192, seed=1), True),
                          ("ER(2048, 0.5) int8", wl.erdos_renyi(2048, 0.5, seed=1), False)):
        dg = D.DeviceGraph(W)
        n = dg.n
        words, g64, Gf, Lf = _local_optimum(dg, 3, spin)
        for _ in range(3):
            dg.double_bit_flips(words, g64, spin, Gf, Lf)
        ms = _timed(lambda: dg.double_bit_flips(words, g64, spin, Gf, Lf), 20)
        pairs = n * (n - 1) // 2
        wbytes = pairs * (1 if dg.is_integer else 4)
        _emit(leg="double", graph=name, n=n, ms_per_pass=round(ms, 4), pairs_per_s=pairs / ms * 1e3,
              w_bytes=wbytes, gbs=round(wbytes / ms / 1e6, 1), hbm_frac=round(wbytes / ms / 1e6 / hbm, 3),
              peak_basis=f"{src} HBM copy bandwidth {hbm} GB/s", l2_flushed=True)


def double_pass_leg():
    """One double-flip pass on SK n=8192 float32 from a single-flip local
    optimum (kernels.cl:150-231 semantics): prep, seed and streaming kernels as
    one call, CUDA events around it, L2 flushed before each of 20 passes. The
    algorithmic bytes are the upper triangle of W (n(n-1)/2 float32)."""
    from pyqrackising_b200 import device as D
    from pyqrackising_b200 import workloads as wl

    hbm, _, src = peaks()
    dg = D.DeviceGraph(wl.sherrington_kirkpatrick(8192, seed=1))
    n = dg.n
    words, g64, Gf, Lf = _local_optimum(dg, 3, True)
    for _ in range(3):
        dg.double_bit_flips(words, g64, True, Gf, Lf)
    ms = _timed(lambda: dg.double_bit_flips(words, g64, True, Gf, Lf), 20)
    wbytes = n * (n - 1) // 2 * 4
    return {
        "workload": "SK n=8192 float32 from a single-flip local optimum, one pass over all pairs, L2 flushed",
        "ms_per_pass": ms,
        "pairs_per_s": n * (n - 1) // 2 / ms * 1e3,
        "w_bytes": wbytes,
        "achieved_GBps": wbytes / ms / 1e6,
        "frac_pass": wbytes / ms / 1e6 / hbm,
        "peak_basis": f"{src} HBM copy bandwidth {hbm} GB/s (the whole pass: prep, seed and stream kernels)",
    }


def leg_gray():
    from pyqrackising_b200 import device as D
    from pyqrackising_b200 import workloads as wl

    mpe = D.max_gpu_proc_elem()
    for name, W, spin, iters, seeds in (
        ("SK n=8192 float32", wl.sherrington_kirkpatrick(8192, seed=1), True, 8192 * 8192, mpe),
        ("ER(1024, 0.5) float32", wl.erdos_renyi(1024, 0.5, seed=1), False, 1024 * 1024 // 16, mpe),
    ):
        import torch

        dg = D.DeviceGraph(W)
        n = dg.n
        words, g64, _, _ = _local_optimum(dg, 4, spin)
        bound = (iters + seeds - 1) // seeds
        for _ in range(2):
            dg.gray(words, g64, spin, bound, seeds)
        ms = _timed(lambda: dg.gray(words, g64, spin, bound, seeds), 5)
        blocks = dg.n64
        positions = sum(((bound - 1 - s) // seeds + 1) * blocks for s in range(seeds) if bound > s)
        _, eout = dg.gray(words, g64, spin, bound, seeds)
        torch.cuda.synchronize()
        _emit(leg="gray", graph=name, n=n, seeds=seeds, iterations=iters, ms_per_search=round(ms, 3),
              positions=positions, positions_per_s=positions / ms * 1e3,
              improving_seeds=int((eout > 0).sum().item()))


def leg_tfim():
    import importlib

    import torch

    from pyqrackising_b200 import device as D
    from pyqrackising_b200 import workloads as wl

    MT = importlib.import_module("pyqrackising_b200.maxcut_tfim")
    for name, W in (("3-regular n=2048 +-1", wl.regular_pm1_fast(2048, seed=5)),
                    ("ER(2048, 0.5)", wl.erdos_renyi(2048, 0.5, seed=1))):
        dg = D.DeviceGraph(W)
        _, _, cum = MT.hamming_cdf(dg, 6, 8.0, 8.0)
        shots = ((max(1, (2048 << 6) >> 1) + 31) >> 5) << 5
        buf = MT.sample_batch(dg, cum, shots, 5.0, 1, 0)
        for r in range(2):
            MT.sample_batch(dg, cum, shots, 5.0, 1, r, out=buf)
        ms = _timed(lambda: MT.sample_batch(dg, cum, shots, 5.0, 1, 7, out=buf), 3, flush=False)
        bits = dg.unpack(buf, rows=shots)
        _emit(leg="tfim_sampler", graph=name, quality=6, shots=shots, ms_per_round=round(ms, 3),
              shots_per_s=shots / ms * 1e3, mean_selected_per_shot=float(bits.sum()) / shots,
              note="W (16 MB) is L2-resident; a selected node is a picked or underflowed weight")
    W1 = wl.erdos_renyi(1024, 0.5, seed=1)
    MT.set_seed(0)
    MT.maxcut_tfim(W1, quality=2)
    runs = []
    for seed in range(5):
        MT.set_seed(seed)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, cut, _ = MT.maxcut_tfim(W1, quality=2)
        torch.cuda.synchronize()
        runs.append((time.perf_counter() - t0, cut))
    MT.set_seed(None)
    _emit(leg="maxcut_tfim", graph="ER(1024, 0.5)", quality=2, wall_s=[round(t, 4) for t, _ in runs],
          cuts=[c for _, c in runs], note="host wall time per call, W upload and preparation included")


def leg_sparse():
    import scipy.sparse as sp
    import torch

    from pyqrackising_b200 import spin_glass_solver, spin_glass_solver_sparse
    from pyqrackising_b200 import workloads as wl

    W = wl.gnp_weighted(16384, 0.01, seed=1, dist="normal")
    G = sp.csr_matrix(np.triu(W, 1))
    best = "".join("1" if b else "0" for b in wl.random_bits(16384, 9))
    out = {}
    for name, fn, arg in (("sparse", spin_glass_solver_sparse, G), ("dense", spin_glass_solver, W)):
        fn(arg, best_guess=best)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, cut, _, energy = fn(arg, best_guess=best)
        torch.cuda.synchronize()
        out[name] = (time.perf_counter() - t0, cut, energy)
    _emit(leg="sparse", graph="G(16384, 0.01) N(0,1)", nnz_upper=int(G.nnz),
          sparse_s=round(out["sparse"][0], 3), dense_s=round(out["dense"][0], 3),
          sparse_energy=out["sparse"][2], dense_energy=out["dense"][2],
          note="same best_guess; host wall time per call, coordinate upload / W upload included")


def leg_bnb():
    import contextlib
    import io
    import re

    from pyqrackising_b200 import solve_maxcut_bnb
    from pyqrackising_b200 import workloads as wl

    warm = solve_maxcut_bnb(wl.regular_pm1_fast(12, seed=3), best_guess="0" * 12, verbose=False)
    assert warm[4]
    for n in (28, 32):
        W = wl.regular_pm1_fast(n, seed=3)
        rng = np.random.default_rng(1)
        guess = "".join("1" if b else "0" for b in rng.random(n) < 0.5)
        for cap in (64, 4096):
            buf = io.StringIO()
            t0 = time.perf_counter()
            with contextlib.redirect_stdout(buf):
                bits, cut, _, _, certified = solve_maxcut_bnb(W, best_guess=guess, verbose=True, batch_size=cap)
            dt = time.perf_counter() - t0
            m = re.search(r"Nodes explored: (\d+)\s+\|\s+Pruned: (\d+)", buf.getvalue())
            _emit(leg="bnb", graph=f"3-regular n={n} +-1", batch_size=cap, wall_s=round(dt, 3), cut=cut,
                  certified=bool(certified), nodes=int(m.group(1)), pruned=int(m.group(2)),
                  nodes_per_s=round(int(m.group(1)) / dt))


def leg_flips(tasks=444, budget=64, fields="f64"):
    import torch

    from pyqrackising_b200 import workloads as wl
    from pyqrackising_b200.batch import BatchedSearch
    from pyqrackising_b200.device import DeviceGraph

    bs = BatchedSearch([DeviceGraph(wl.sherrington_kirkpatrick(8192, seed=1))])
    tg = torch.zeros(tasks, dtype=torch.int32, device="cuda")
    w0 = bs.random_states(np.zeros(tasks, dtype=np.int32), seed=5)
    for _ in range(2):
        v, _, flips, st = bs.run(tg, w0, True, rounds=0, flip_budget=budget, fields=fields)
    torch.cuda.synchronize()
    _emit(leg="flips", tasks=tasks, flip_budget=budget, fields=fields, flips=int(flips.item()), status=int(st.item()))
    if int(st.item()) not in (0, 3):  # 3: the flip budget ran out, as intended
        raise SystemExit(1)


def leg_cluster(n=8192, starts=8):
    import torch

    from pyqrackising_b200 import workloads as wl
    from pyqrackising_b200.batch import BatchedSearch
    from pyqrackising_b200.device import DeviceGraph

    bs = BatchedSearch([DeviceGraph(wl.sherrington_kirkpatrick(n, seed=1))])
    tasks = [0] * starts
    w0 = bs.random_states(tasks, seed=7)
    v, best, flips, st = bs.cluster_ascent(tasks, w0, True, cluster_size=8)
    # the cluster form keeps float64 fields: compare with the CTA form's float64 fields
    v2, best2, flips2, st2 = bs.run(tasks, w0, True, rounds=0, fields="f64")
    torch.cuda.synchronize()
    ok = torch.equal(best, best2) and int(st.item()) == 0
    _emit(leg="cluster", flips=int(flips.item()), best=float(v.max()), matches_batched=ok)
    if not ok:
        raise SystemExit(1)


def leg_mpnn(n=16384):
    import torch

    from pyqrackising_b200 import learned as L
    from pyqrackising_b200 import workloads as wl
    from pyqrackising_b200.device import DeviceGraph

    dg = DeviceGraph(wl.gnp_weighted(n, 0.01, seed=5, dist="normal"))
    ctx = L.GraphContext(dg)
    net = L.ProposalNet(seed=1)
    F = ctx.features(dg.pack(np.random.default_rng(1).random(n) < 0.5))
    logits, cache = net.forward(ctx, F)
    _, dl, _ = net.loss_grad(logits, torch.full((n,), 1.0 / n, device="cuda"))
    net.backward(ctx, cache, dl)
    torch.cuda.synchronize()
    ok = bool(torch.isfinite(logits).all().item()) and bool(torch.isfinite(net.g).all().item())
    _emit(leg="mpnn", n=n, finite=ok)
    if not ok:
        raise SystemExit(1)


def leg_csr(n=200000, p=1e-4):
    """A sparse graph too large for the dense form, on compressed rows:
    G(n, p) with N(0,1) weights (G(200000, 1e-4): 160 GB as a dense float32
    matrix). spin_glass_solver_sparse from a random best_guess (host wall time,
    rows built and uploaded inside), then the compressed-row double pass and
    one descent timed alone (CUDA events)."""
    import scipy.sparse as sp
    import torch

    from oracle import oracle as O
    from pyqrackising_b200 import spin_glass_solver_sparse
    from pyqrackising_b200.sparse import SparseDeviceGraph, use_compressed_rows

    rng = np.random.default_rng(9)
    m = int(n * (n - 1) / 2 * p)
    r = rng.integers(0, n, size=2 * m)
    c = rng.integers(0, n, size=2 * m)
    keep = r < c
    r, c = r[keep][:m], c[keep][:m]
    U = sp.coo_matrix((rng.standard_normal(len(r)).astype(np.float32), (r, c)), shape=(n, n)).tocsr()
    U.sum_duplicates()
    guess = "".join("1" if b else "0" for b in rng.random(n) < 0.5)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    bits, cut, _, energy = spin_glass_solver_sparse(U, best_guess=guess)
    torch.cuda.synchronize()
    t_solve = time.perf_counter() - t0
    sg = SparseDeviceGraph(U)
    words = sg.pack(np.array([b == "1" for b in bits]))
    _, g64 = sg.gains(words)
    G, L = O.flip_geometry(n, 148)
    sg.double_bit_flips(words, g64, True, G, L)
    ms_double = _timed(lambda: sg.double_bit_flips(words, g64, True, G, L), 3, flush=False)
    start = sg.pack(rng.random(n) < 0.5)
    _, gs = sg.gains(start)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    _, fl, rc = sg.single_descent(start, gs, True, G, L, 1 << 20)
    b.record()
    b.synchronize()
    ms_desc = a.elapsed_time(b)
    flips = int(fl.item())
    _emit(leg="csr", graph=f"G({n}, {p}) N(0,1) float32", nnz=sg.nnz, dense_bytes=4 * n * n,
          compressed_row_bytes=int(sg.nnz * 8 + (n + 1) * 8), uses_compressed_rows=use_compressed_rows(n),
          solve_s=round(t_solve, 3), energy=energy, cut=cut,
          double_pass_ms=round(ms_double, 3), pairs_per_s=n * (n - 1) / 2 / (ms_double / 1e3),
          descent_ms=round(ms_desc, 2), descent_flips=flips, us_per_flip=round(1e3 * ms_desc / max(flips, 1), 3))


LEGS = {"csr": leg_csr, "double": leg_double, "gray": leg_gray, "tfim": leg_tfim, "sparse": leg_sparse, "bnb": leg_bnb,
        "flips": leg_flips, "cluster": leg_cluster, "mpnn": leg_mpnn}


def make_graph():
    from pyqrackising_b200 import workloads as wl

    return wl.erdos_renyi(N_NODES, EDGE_P, seed=1)


def make_batch(seed, rows=BATCH):
    """Candidates of batch `seed` (seeded uniform bits); the first `rows` rows
    of the full batch."""
    return np.random.default_rng(1000 + seed).random((rows, N_NODES)) < 0.5


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--no-ttb", action="store_true", help="skip the SK n=8192 time-to-best leg")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-uneven and flip-bandwidth legs")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--leg", nargs="+", choices=sorted(LEGS), help="run only these legs (one GPU), one JSON line each")
    ap.add_argument("--leg-args", nargs="*", default=[], help="positional arguments of a single leg (flips: tasks budget f64|f32)")
    args = ap.parse_args()
    if args.leg:
        import torch

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        for name in args.leg:
            conv = [int(a) if a.lstrip("-").isdigit() else a for a in args.leg_args]
            LEGS[name](*conv)
        return 0

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = dist_mod

    from oracle import oracle as O
    from pyqrackising_b200 import _lib
    from pyqrackising_b200.device import DeviceGraph

    W = make_graph()
    dg = DeviceGraph(W)
    G, L = O.cut_geometry(BATCH, 148)
    nb = 2
    batches_host = [O.pack32(make_batch(rank * 97 + i)) for i in range(nb)]
    batches = [torch.from_numpy(b.view(np.int32).reshape(-1)).to(dg.device) for b in batches_host]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dg.device)
    stream = torch.cuda.current_stream()

    # correctness spot check against the oracle on a few candidates (outside timing)
    e, be, bi = dg.calculate_cut(batches[0], BATCH, False, G, L)
    pick = np.r_[0:8, BATCH - 8:BATCH]
    ref = O.cut_values(W, batches_host[0][pick], len(pick), 0)
    assert np.array_equal(e.cpu().numpy()[pick], ref), "scoring mismatch against the oracle"

    for i in range(args.warmup):
        dg.calculate_cut(batches[i % nb], BATCH, False, G, L, energies=False)
    torch.cuda.synchronize()

    # device-resident timing: events around each step, L2 flushed between steps;
    # the library also records events around the scoring GEMM launch itself
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clocks:
        clocks.wait_first()
        wall0 = time.perf_counter()
        for i in range(args.steps):
            flush.fill_(i & 0xFF)
            evs[i][0].record(stream)
            kev[i][0].record(stream)  # materialise the events before handing them over
            kev[i][1].record(stream)
            _lib.load().pqi_score_set_events(ctypes.c_void_p(kev[i][0].cuda_event), ctypes.c_void_p(kev[i][1].cuda_event))
            dg.calculate_cut(batches[i % nb], BATCH, False, G, L, energies=False)
            evs[i][1].record(stream)
        _lib.load().pqi_score_set_events(None, None)
        torch.cuda.synchronize()
        wall = time.perf_counter() - wall0
        step_ms = [a.elapsed_time(b) for a, b in evs]
        kernel_ms = float(np.mean([a.elapsed_time(b) for a, b in kev]))
        total_ms = float(np.sum(step_ms))

        # e2e through the C ABI with host buffers (pinned), copies inside the
        # window: each step copies its packed batch host -> device on a copy
        # stream (double-buffered, so step i+1's copy overlaps step i's
        # scoring), scores it, and reads the (value, index) pair back.
        e2e_ms = e2e_pipeline(dg, batches_host, batches[0], G, L, args.steps, args.warmup)
    # the slowest rank's device time; then the batches' best candidate over
    # ranks (each rank scored its own share of the candidates): one exchange
    from pyqrackising_b200 import distributed as DI

    cdev = DI.collective_device(dist)
    total_ms = DI.max_over_ranks(total_ms, dist, cdev)
    e2e_ms = DI.max_over_ranks(e2e_ms, dist, cdev)
    _, be, bi = dg.calculate_cut(batches[0], BATCH, False, G, L, energies=False)
    win_words = batches[0].view(BATCH, -1)[int(bi.item())]
    best_value, best_rank, _ = DI.best_over_ranks(float(be.item()), win_words, dist, cdev)

    ms_per_step = total_ms / args.steps
    value = world * BATCH * args.steps / (total_ms / 1000.0)
    e2e_value = world * BATCH * args.steps / (e2e_ms / 1000.0)
    hbm, bf16, src = peaks()
    ops = 2.0 * BATCH * N_NODES * N_NODES
    achieved = ops / (kernel_ms / 1000.0) / 1e12
    int8_peak = 2.0 * bf16
    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int8" if dg.is_integer else "bf16x2",
        "data": "synthetic",
        "config": workload_config(),
        "e2e": {
            "value": e2e_value,
            "unit": UNIT,
            "h2d_bytes_per_step": int(batches_host[0].nbytes),
            "d2h_bytes_per_step": 8,
            "ms_per_step": e2e_ms / args.steps,
            "h2d_only_ms_per_step": getattr(e2e_pipeline, "h2d_only_ms", float("nan")) / args.steps,
        },
        "roofline": {
            "bound": "tensor",
            "achieved": achieved,
            "peak": int8_peak,
            "unit": "TFLOP/s",
            "frac": achieved / int8_peak,
            "ops_note": "int8 multiply-adds counted as 2 ops (TOPS)",
            # dram__bytes_read.sum + dram__bytes_write.sum of one launch of this
            # workload (profiles/score_tc_kernel_er2048_b65536.md)
            "traffic": 196.3e6,
            "traffic_unit": "bytes per launch (ncu)",
            "algorithmic_bytes_per_launch": float(BATCH * N_NODES + N_NODES * N_NODES + BATCH * N_NODES // 8),
            "peak_basis": f"int8 dense = 2 x bf16 dense ({src} bf16 {bf16} TFLOP/s)",
            "kernel": "score_tc_kernel<int8> (tcgen05 GEMM + row-dot epilogue), CUDA events around the launch",
            "kernel_ms": kernel_ms,
            "algorithmic_ops_per_launch": ops,
            # the whole step (expansion pass, GEMM, selection) against the same peak
            "frac_step": ops / (ms_per_step / 1000.0) / 1e12 / int8_peak,
        },
        # per step: score_tc_kernel (the L2 flush is torch's fill)
        # per step the library launches the +-1 expansion and the scoring GEMM
        # (the zeroing of its selection words is a memset, not a kernel)
        "gpu_launches": 2 * args.steps,
        "best_over_ranks": {"value": best_value, "rank": best_rank},
        "wall_s_timed_loop": wall,
    }
    if rank == 0:
        line["clocks"] = clocks.summary()
        if world == 1:
            line["scoring_b4096"] = scoring_batch_leg(dg)
        if world == 1 and not args.no_ttb:
            line["time_to_best"] = time_to_best()
            line["time_to_best_learned"] = time_to_best_learned()
        if world == 1 and not args.no_batched:
            line["plain_small"] = plain_small_leg()
            line["batched"] = batched_leg()
            line["learned"] = learned_leg()
            line["flip_updates"] = flip_bandwidth_leg()
            line["flip_updates_f32_fields"] = flip_bandwidth_leg(fields="f32")
            try:
                line["double_pass"] = double_pass_leg()
            except Exception as ex:  # pragma: no cover
                line["double_pass"] = {"unavailable": str(ex)}
        if world == 1:
            try:
                line["cpu_baseline"] = cpu_baseline(W, make_batch(0, 2048))
            except Exception as ex:  # pragma: no cover
                line["cpu_baseline"] = {"unavailable": str(ex)}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
