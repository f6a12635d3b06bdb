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
``spin_glass_solver`` (the fallback and the judge: every value is the
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


def train_streaming(net: L.ProposalNet, count: int = 10000, chunk: int = 64, seed: int = 0,
                    tasks_per_graph: int = 4, rounds: int = 8, lr: float = 2e-3, batch: int = 16,
                    log=None):
    """One pass over `count` streamed graphs; returns (loss history, examples seen)."""
    hist, seen = [], 0
    t0 = time.time()
    for c0 in range(0, count, chunk):
        Ws = [wl.proposal_training_graph(i, seed=seed) for i in range(c0, min(count, c0 + chunk))]
        dgs = [DeviceGraph(W) for W in Ws]
        ex = L.make_examples(dgs, tasks_per_graph=tasks_per_graph, rounds=rounds, seed=seed + c0)
        if ex:
            hist += L.train(net, dgs, ex, epochs=1, lr=lr, batch=batch)
            seen += len(ex)
        del dgs
        if log is not None:
            log(f"graphs {min(count, c0 + chunk)}/{count} examples {seen} "
                f"loss {np.mean(hist[-8:]) if hist else float('nan'):.4f} ({time.time() - t0:.0f} s)")
    return hist, seen


def ils_compare(net: L.ProposalNet | None, dg: DeviceGraph, starts: int = 32, rounds: int = 8,
                kick: int | None = None, seed: int = 0, spin: bool = True, temperature: float = 3.0):
    """Uniform-kick vs proposal-kick iterated search from the same ascent
    states (same seeds, same budget). Returns a dict of values and times."""
    bs = BatchedSearch([dg])
    tg = [0] * starts
    w0 = bs.random_states(tg, seed=seed)
    k = kick if kick is not None else max(2, dg.n // 16)
    torch.cuda.synchronize()
    t = time.perf_counter()
    vA, wA, _, _ = bs.run(tg, w0, spin, rounds=0)
    torch.cuda.synchronize()
    t_ascent = time.perf_counter() - t
    A = wA.reshape(-1).contiguous()
    t = time.perf_counter()
    vU, _, _, sU = bs.run(tg, A, spin, rounds=rounds, kick=k, seed=seed + 1)
    torch.cuda.synchronize()
    t_uniform = time.perf_counter() - t
    out = {"n": dg.n, "starts": starts, "rounds": rounds, "kick": k,
           "ascent_best": float(vA.max()), "ascent_s": t_ascent,
           "uniform_best": float(vU.max()), "uniform_mean": float(vU.mean()), "uniform_s": t_uniform}
    if net is not None:
        t = time.perf_counter()
        cdf, off = L.task_proposals(net, dg, wA, temperature=temperature)
        bsT = BatchedSearch([dg] * starts)  # one descriptor (and proposal) per task
        vP, _, _, sP = bsT.run(list(range(starts)), A, spin, rounds=rounds, kick=k, seed=seed + 1,
                               kick_cdf=cdf, cdf_offset=off)
        torch.cuda.synchronize()
        out.update({"learned_best": float(vP.max()), "learned_mean": float(vP.mean()),
                    "learned_s": time.perf_counter() - t, "temperature": temperature})
    return out


def evaluate(net: L.ProposalNet | None, n: int = 16384, p: float = 0.01, seed: int = 5,
             starts: int = 32, rounds: int = 8):
    """The evaluation graph: plain local search (judge and fallback) next to the
    uniform- and proposal-kick batched searches."""
    SG = importlib.import_module("pyqrackising_b200.spin_glass_solver")
    W = wl.gnp_weighted(n, p, seed=seed, dist="normal")
    dg = DeviceGraph(W)
    start = np.random.default_rng(seed).random(n) < 0.5
    SG.local_search(dg, start, True, 4 * n, 148, 148, 0.0)  # warm
    torch.cuda.synchronize()
    t = time.perf_counter()
    words, _ = SG.local_search(dg, start, True, 4 * n, 148, 148, 0.0)
    _, e = dg.rescore(words)
    torch.cuda.synchronize()
    res = {"graph": f"G({n},{p}) N(0,1) float32", "plain_energy": float(e.item()),
           "plain_s": time.perf_counter() - t}
    res.update(ils_compare(net, dg, starts=starts, rounds=rounds, seed=seed))
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
    hist, seen = train_streaming(net, count=args.graphs, chunk=args.chunk, seed=args.seed,
                                 log=lambda m: print(m, flush=True))
    if args.out:
        net.save(args.out)
    print(json.dumps({"graphs": args.graphs, "examples": seen, "steps": len(hist),
                      "loss_first": float(np.mean(hist[:16])), "loss_last": float(np.mean(hist[-16:]))}), flush=True)


if __name__ == "__main__":
    main()
