"""Golden tours of the reference's TSP heuristic, made by importing the
reference itself (build container only):

    NUMBA_CACHE_DIR=/tmp/numba_cache python tests/golden/make_tsp_golden.py

Each case seeds the random stream of the reference's compiled helpers
(numba's generator, seeded from inside a compiled function) and runs
``tsp_symmetric`` / ``tsp_asymmetric`` (pyqrackising/tsp.py:686,1005) with
``monte_carlo=True`` (random splits, no solver calls) on a seeded instance:
Euclidean distances for the symmetric cases, uniform random weights for the
asymmetric ones, several sizes (brute force below 7 cities, recursion above)
and the start/end/cyclic/k_neighbors options. ``tests/test_tsp.py`` replays
every case through ``pyqrackising_b200.tsp`` with the same seed and checks the
tour and its weight (the instances are rebuilt there from the same seeds).
Writes ``tests/golden/golden_tsp.npz``.
"""

from __future__ import annotations

import importlib
import json
import os
import sys

import numpy as np

REFERENCE = os.environ.get("PQI_REFERENCE_ROOT", "/root/reference")
sys.path.insert(0, REFERENCE)
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache")

from numba import njit  # noqa: E402


@njit
def _seed(s):
    np.random.seed(s)


def instance(kind, n, seed):
    rng = np.random.default_rng(1000 + 17 * n + seed)
    if kind == "sym":
        P = rng.random((n, 2))
        return np.sqrt(((P[:, None, :] - P[None, :, :]) ** 2).sum(-1))
    W = rng.random((n, n))
    np.fill_diagonal(W, 0.0)
    return W


CASES = []
for n in (2, 3, 4, 5, 6, 7, 8, 9, 12, 17, 25, 40):
    for kind in ("sym", "asym"):
        CASES.append({"kind": kind, "n": n, "seed": 1, "kw": {}})
        CASES.append({"kind": kind, "n": n, "seed": 2, "kw": {"is_cyclic": False}})
        if n >= 3:
            CASES.append({"kind": kind, "n": n, "seed": 3, "kw": {"is_cyclic": False, "start_node": 1}})
            CASES.append({"kind": kind, "n": n, "seed": 4, "kw": {"is_cyclic": False, "start_node": 0, "end_node": n - 1}})
            CASES.append({"kind": kind, "n": n, "seed": 5, "kw": {"is_cyclic": False, "end_node": 2}})
            CASES.append({"kind": kind, "n": n, "seed": 6, "kw": {"start_node": 2}})
        CASES.append({"kind": kind, "n": n, "seed": 7, "kw": {"k_neighbors": 0}})
        CASES.append({"kind": kind, "n": n, "seed": 8, "kw": {"k_neighbors": 5}})
for n in (60, 90):
    for kind in ("sym", "asym"):
        CASES.append({"kind": kind, "n": n, "seed": 9, "kw": {}})


def main():
    tsp = importlib.import_module("pyqrackising.tsp")
    out = {"cases": json.dumps(CASES)}
    for i, case in enumerate(CASES):
        G = instance(case["kind"], case["n"], case["seed"])
        fn = tsp.tsp_symmetric if case["kind"] == "sym" else tsp.tsp_asymmetric
        _seed(case["seed"])
        path, weight = fn(G, **case["kw"])
        out[f"path{i}"] = np.asarray([int(x) for x in path], dtype=np.int64)
        out[f"weight{i}"] = np.float64(weight)
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_tsp.npz"), **out)


if __name__ == "__main__":
    main()
