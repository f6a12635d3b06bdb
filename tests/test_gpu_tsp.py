"""TSP with MAXCUT splits on the device (monte_carlo=False): one batched
launch per recursion depth, or the solver drop-in per subgraph."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _euclid(n, seed):
    P = np.random.default_rng(seed).random((n, 2))
    return np.sqrt(((P[:, None, :] - P[None, :, :]) ** 2).sum(-1))


def _cut(G, a, b):
    return float(G[np.ix_(a, b)].sum())


@pytest.mark.parametrize("n", [40, 150])
def test_batched_splits_one_launch_per_depth(n, monkeypatch):
    from pyqrackising_b200 import batch, tsp

    launches = []
    orig = batch.BatchedSolver.step

    def counted(self):
        launches.append(len(self.graphs))
        return orig(self)

    monkeypatch.setattr(batch.BatchedSolver, "step", counted)
    G = _euclid(n, 3)
    table = tsp._plan_batched(G, list(range(n)), n, None, None, True, True,
                              {"multi_start": 1, "seed": 0, "quality": None, "shots": None,
                               "anneal_t": None, "anneal_h": None, "repulsion_base": None})
    depth = max(len(k) for k in table) + 1
    assert len(launches) == depth and launches[0] == 1
    assert sum(launches) == len(table)
    # every split is a non-trivial partition, and the root's cut beats random ones
    a, b = table[""]
    assert a and b and sorted(a + b) == list(range(n))
    rng = np.random.default_rng(0)
    rand = [rng.random(n) < 0.5 for _ in range(64)]
    best_random = max(_cut(G, np.nonzero(~m)[0], np.nonzero(m)[0]) for m in rand)
    assert _cut(G, a, b) > best_random

    for kind in ("sym", "asym"):
        W = G if kind == "sym" else G + 0.1 * np.random.default_rng(1).random((n, n))
        if kind == "asym":
            np.fill_diagonal(W, 0.0)
        fn = tsp.tsp_symmetric if kind == "sym" else tsp.tsp_asymmetric
        tsp.seed(5)
        p1, w1 = fn(W, monte_carlo=False)
        tsp.seed(5)
        p2, w2 = fn(W, monte_carlo=False)
        assert p1 == p2 and w1 == w2  # seeded splits and re-splits: the same tour
        assert p1[0] == p1[-1] and sorted(p1[:-1]) == list(range(n))
        assert w1 == pytest.approx(sum(W[x, y] for x, y in zip(p1, p1[1:])), rel=1e-12)


def test_solver_splits_per_subgraph():
    """split='solver': the spin_glass_solver drop-in per subgraph (the
    reference's call), a valid tour."""
    from pyqrackising_b200 import tsp

    G = _euclid(24, 7)
    tsp.seed(1)
    path, w = tsp.tsp_symmetric(G, monte_carlo=False, split="solver", quality=2)
    assert path[0] == path[-1] and sorted(path[:-1]) == list(range(24))
    assert w == pytest.approx(sum(G[x, y] for x, y in zip(path, path[1:])), rel=1e-12)
