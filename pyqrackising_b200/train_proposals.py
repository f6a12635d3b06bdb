"""Training and evaluation of the flip-proposal network on streamed graphs.

Training stream: graphs i = 0 .. count-1 of
``workloads.proposal_training_graph`` (n ~ U[128, 2048]; even i 3-regular
+-1, odd i G(n, 0.05) with N(0, 1) weights), taken in chunks: each chunk's
graphs are prepared on the GPU, the batched search generates the examples
(local optimum A, the nodes where a better optimum B found by iterated search
differs), the network takes one Adam pass over them, and the chunk is dropped.

Evaluation: one graph (default G(16384, 0.01) with N(0, 1) weights); from the
same starting states, the batched iterated search with uniform kicks and with
kicks drawn from the network's proposal, next to the plain local search of
``spin_glass_solver`` (the fallback and the arbiter: every value is the
search's exact bookkeeping, re-scored in float64).

    python -m pyqrackising_b200.train_proposals --graphs 10000 --out net.pt
    python -m pyqrackising_b200.train_proposals --eval net.pt
"""

from __future__ import annotations

import argparse
import importlib
import json
import time

import numpy as np
import torch

from . import learned as L
from . import workloads as wl
from .batch import BatchedSearch
from .device import DeviceGraph


def lr_schedule(peak: float, total_steps: int, warmup: int = 50, floor: float = 0.1):
    """Linear warm-up to `peak`, then cosine decay to `floor` * peak."""
    import math

    def lr(step):
        if step < warmup:
            return peak * (step + 1) / warmup
        t = min(1.0, (step - warmup) / max(1, total_steps - warmup))
        return peak * (floor + (1 - floor) * 0.5 * (1 + math.cos(math.pi * t)))

    return lr


def train_streaming(net: L.ProposalNet, count: int = 10000, chunk: int = 64, seed: int = 0,
                    tasks_per_graph: int = 4, rounds: int = 8, lr: float = 5e-4, batch: int = 16,
                    log=None, check_every: int = 0, check_graphs=None):
    """One pass over `count` streamed graphs; returns (loss history, examples
    seen). The learning rate warms up and decays over the expected number of
    optimiser steps. Every `check_every` graphs the held-out gain of the
    proposals over uniform kicks is measured on `check_graphs`: the best
    parameters so far are kept (and restored at the end), and a network whose
    proposals have gone uniform (dead units: zero gain on every check graph)
    is restored to the best parameters with Adam reset and the rate halved."""
    hist, seen = [], 0
    scale = [1.0]
    base = lr_schedule(lr, total_steps=max(100, count * 3 // batch))
    sched = lambda step: scale[0] * base(step)  # noqa: E731
    best_gain, best_params = -float("inf"), None
    t0 = time.time()
    for c0 in range(0, count, chunk):
        Ws = [wl.proposal_training_graph(i, seed=seed) for i in range(c0, min(count, c0 + chunk))]
        dgs = [DeviceGraph(W) for W in Ws]
        ex = L.make_examples(dgs, tasks_per_graph=tasks_per_graph, rounds=rounds, seed=seed + c0)
        if ex:
            hist += L.train(net, dgs, ex, epochs=1, lr=sched, batch=batch)
            seen += len(ex)
        del dgs
        done = min(count, c0 + chunk)
        msg = (f"graphs {done}/{count} examples {seen} step {net.step_count} "
               f"loss {np.mean(hist[-8:]) if hist else float('nan'):.4f} ({time.time() - t0:.0f} s)")
        last = done == count
        if check_every and check_graphs and (last or (done // check_every) != ((done - chunk) // check_every)):
            gains = [r["learned_mean"] - r["uniform_mean"]
                     for r in (ils_compare(net, dg, starts=32, rounds=8, seed=7) for dg in check_graphs)]
            g = float(np.mean(gains))
            msg += f" held-out gains {[round(x, 2) for x in gains]}"
            if all(x == 0.0 for x in gains) and best_params is not None:
                net.restore(best_params)
                scale[0] *= 0.5
                msg += f" (dead: restored best, rate x{scale[0]:g})"
            elif g > best_gain:
                best_gain, best_params = g, net.snapshot()
        if log is not None:
            log(msg)
    if best_params is not None:
        net.restore(best_params, reset_moments=False)
    return hist, seen


def ils_compare(net: L.ProposalNet | None, dg: DeviceGraph, starts: int = 32, rounds: int = 8,
                kick: int | None = None, seed: int = 0, spin: bool = True, temperature: float = 3.0,
                keep_states: bool = False):
    """Uniform-kick vs proposal-kick iterated search from the same ascent
    states (same seeds, same budget). Returns a dict of values and times."""
    bs = BatchedSearch([dg])
    tg = [0] * starts
    w0 = bs.random_states(tg, seed=seed)
    k = kick if kick is not None else max(2, min(dg.n // 16, 64))
    torch.cuda.synchronize()
    t = time.perf_counter()
    vA, wA, _, _ = bs.run(tg, w0, spin, rounds=0)
    torch.cuda.synchronize()
    t_ascent = time.perf_counter() - t
    A = wA.reshape(-1).contiguous()
    t = time.perf_counter()
    vU, wU, _, sU = bs.run(tg, A, spin, rounds=rounds, kick=k, seed=seed + 1)
    torch.cuda.synchronize()
    t_uniform = time.perf_counter() - t
    out = {"n": dg.n, "starts": starts, "rounds": rounds, "kick": k,
           "ascent_best": float(vA.max()), "ascent_s": t_ascent,
           "uniform_best": float(vU.max()), "uniform_mean": float(vU.mean()), "uniform_s": t_uniform}
    if net is not None:
        t = time.perf_counter()
        cdf, off = L.task_proposals(net, dg, wA, temperature=temperature)
        bsT = BatchedSearch([dg] * starts)  # one descriptor (and proposal) per task
        vP, wP, _, sP = bsT.run(list(range(starts)), A, spin, rounds=rounds, kick=k, seed=seed + 1,
                                kick_cdf=cdf, cdf_offset=off)
        torch.cuda.synchronize()
        out.update({"learned_best": float(vP.max()), "learned_mean": float(vP.mean()),
                    "learned_s": time.perf_counter() - t, "temperature": temperature})
    if keep_states:
        states = {"uniform": bs.unpack(wU[int(torch.argmax(vU).item())].unsqueeze(0), [0])[0]}
        if net is not None:
            states["learned"] = bs.unpack(wP[int(torch.argmax(vP).item())].unsqueeze(0), [0])[0]
        out["states"] = states
    return out


def evaluate(net: L.ProposalNet | None, n: int = 16384, p: float = 0.01, seed: int = 5,
             starts: int = 32, rounds: int = 8):
    """The evaluation graph. The batched iterated search runs with uniform and
    with proposal kicks from the same ascent optima; the plain local search of
    spin_glass_solver is the arbiter and the refiner: it runs from a random start
    and from each search's best state, and every value is float64 re-scoring."""
    SG = importlib.import_module("pyqrackising_b200.spin_glass_solver")
    W = wl.gnp_weighted(n, p, seed=seed, dist="normal")
    dg = DeviceGraph(W)
    start = np.random.default_rng(seed).random(n) < 0.5

    def plain_from(bits):
        torch.cuda.synchronize()
        t = time.perf_counter()
        words, _ = SG.local_search(dg, bits, True, 4 * n, 148, 148, 0.0)
        _, e = dg.rescore(words)
        torch.cuda.synchronize()
        return float(e.item()), time.perf_counter() - t

    plain_from(start)  # warm
    e_plain, t_plain = plain_from(start)
    res = {"graph": f"G({n},{p}) N(0,1) float32", "plain_energy": e_plain, "plain_s": t_plain}
    r = ils_compare(net, dg, starts=starts, rounds=rounds, seed=seed, keep_states=True)
    states = r.pop("states")
    res.update(r)
    for tag in ("uniform", "learned"):
        if tag in states:
            e, t = plain_from(states[tag])
            res[f"{tag}_then_plain_energy"] = e
            res[f"{tag}_then_plain_s"] = res[f"{tag}_s"] + res["ascent_s"] + t
    if "learned" in states:
        # both kick streams from the same optima, each refined, best kept: the
        # learned starts add to the uniform ones rather than replace them
        res["both_then_plain_energy"] = max(res["uniform_then_plain_energy"], res["learned_then_plain_energy"])
        res["both_then_plain_s"] = res["uniform_then_plain_s"] + res["learned_then_plain_s"] - res["ascent_s"]
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--graphs", type=int, default=10000)
    ap.add_argument("--chunk", type=int, default=64)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=None, help="save the trained network here")
    ap.add_argument("--eval", default=None, help="evaluate a saved network")
    ap.add_argument("--eval-n", type=int, default=16384)
    args = ap.parse_args()
    if args.eval:
        net = L.ProposalNet.load(args.eval)
        print(json.dumps(evaluate(net, n=args.eval_n)), flush=True)
        return
    net = L.ProposalNet(seed=args.seed)
    check = [DeviceGraph(wl.gnp_weighted(400, 0.05, seed=1001, dist="normal")),
             DeviceGraph(wl.regular_pm1_np(400, seed=2001))]
    hist, seen = train_streaming(net, count=args.graphs, chunk=args.chunk, seed=args.seed,
                                 log=lambda m: print(m, flush=True), check_every=1000, check_graphs=check)
    if args.out:
        net.save(args.out)
    print(json.dumps({"graphs": args.graphs, "examples": seen, "steps": len(hist),
                      "loss_first": float(np.mean(hist[:16])), "loss_last": float(np.mean(hist[-16:]))}), flush=True)


if __name__ == "__main__":
    main()
