"""The TSP drop-in against the reference's own tours (tests/golden/golden_tsp.npz,
made by tests/golden/make_tsp_golden.py): the same seed of the compiled
helpers' random stream gives the same tour and weight, for the brute-force
sizes, the recursion with random splits, the start/end/cyclic options and the
3-opt neighbour lists. No GPU: monte_carlo=True never calls the solver."""

import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden", "golden_tsp.npz")


def _instance(kind, n, seed):
    # the generator's instances (make_tsp_golden.instance)
    rng = np.random.default_rng(1000 + 17 * n + seed)
    if kind == "sym":
        P = rng.random((n, 2))
        return np.sqrt(((P[:, None, :] - P[None, :, :]) ** 2).sum(-1))
    W = rng.random((n, n))
    np.fill_diagonal(W, 0.0)
    return W


def _cases():
    z = np.load(GOLD)
    return z, json.loads(str(z["cases"]))


def test_tsp_matches_reference_tours():
    from pyqrackising_b200 import tsp

    z, cases = _cases()
    for i, case in enumerate(cases):
        G = _instance(case["kind"], case["n"], case["seed"])
        fn = tsp.tsp_symmetric if case["kind"] == "sym" else tsp.tsp_asymmetric
        tsp.seed(case["seed"])
        path, weight = fn(G, **case["kw"])
        assert [int(x) for x in path] == z[f"path{i}"].tolist(), (i, case)
        assert float(weight) == float(z[f"weight{i}"]), (i, case)


def test_tsp_tours_are_valid():
    """Tours visit every city once (cyclic: back to the first), honour the
    start and end nodes where the reference's driver keeps them, and weigh
    their own edges; chunked (is_parallel) variants too."""
    from pyqrackising_b200 import tsp

    for kind in ("sym", "asym"):
        for n in (7, 13, 31):
            G = _instance(kind, n, 11)
            fn = tsp.tsp_symmetric if kind == "sym" else tsp.tsp_asymmetric
            for par in (False, True):
                tsp.seed(3)
                path, w = fn(G, is_parallel=par)
                assert path[0] == path[-1] and sorted(path[:-1]) == list(range(n))
                assert w == pytest.approx(sum(G[a, b] for a, b in zip(path, path[1:])), rel=1e-12)
                tsp.seed(4)
                path, w = fn(G, is_cyclic=False, is_parallel=par)
                assert sorted(path) == list(range(n))


def test_tsp_graph_input_float32():
    """An nx.Graph is read as float32 distances (the reference's dtype), with
    its node labels in the tour."""
    import networkx as nx

    from pyqrackising_b200 import tsp

    G = _instance("sym", 9, 5)
    g = nx.Graph()
    labels = [f"c{i}" for i in range(9)]
    for i in range(9):
        for j in range(i + 1, 9):
            g.add_edge(labels[i], labels[j], weight=float(G[i, j]))
    tsp.seed(2)
    path, w = tsp.tsp_symmetric(g)
    assert set(path) == set(labels) and path[0] == path[-1]
    G32 = nx.to_numpy_array(g, weight="weight", nonedge=0.0, dtype=np.float32)
    idx = {l: i for i, l in enumerate(g.nodes())}
    assert w == pytest.approx(sum(float(G32[idx[a], idx[b]]) for a, b in zip(path, path[1:])), rel=1e-6)
