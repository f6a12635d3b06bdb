"""Seeded synthetic instances with the shapes of the five named workloads.

All generators return dense float32 symmetric couplings with a zero diagonal,
the layout ``nx.to_numpy_array(G, weight="weight", nonedge=0.0, dtype=float32)``
gives the reference solver (``pyqrackising/spin_glass_solver.py:458-461``).

* ``regular_pm1`` - random 3-regular graph with +-1 couplings. With n=64 and
  seed 42 this is exactly the reference README generator
  (``scripts/spin_glass.py:10-16``): ``np.random.seed(seed)``, networkx
  ``random_regular_graph(3, n, seed)``, then ``np.random.choice([-1, 1])`` per
  edge in ``G.edges()`` order.
* ``erdos_renyi`` - G(n, p) with unit weights (dense unweighted MAXCUT).
* ``sherrington_kirkpatrick`` - complete graph, J_ij ~ N(0,1)/sqrt(n).
* ``gnp_weighted`` - G(n, p) with weights uniform in (0, 1] or N(0, 1).
* ``batched_uneven`` - a list of instances with n uniform in [lo, hi]: half
  3-regular +-1, half G(n, 0.1) with uniform (0, 1] weights.

Large G(n, p) instances are drawn with numpy (upper triangle Bernoulli) rather
than networkx, which takes minutes at n = 16384.
"""

from __future__ import annotations

import numpy as np


def _symmetrize(upper: np.ndarray) -> np.ndarray:
    u = np.triu(upper, 1)
    w = u + u.T
    return np.ascontiguousarray(w, dtype=np.float32)


def regular_pm1(n: int = 64, seed: int = 42, degree: int = 3) -> np.ndarray:
    import networkx as nx

    np.random.seed(seed)
    G = nx.random_regular_graph(d=degree, n=n, seed=seed)
    for u, v in G.edges():
        G[u][v]["weight"] = np.random.choice([-1, 1])
    return nx.to_numpy_array(G, weight="weight", nonedge=0.0, dtype=np.float32)


def erdos_renyi(n: int = 2048, p: float = 0.5, seed: int = 1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    A = (rng.random((n, n), dtype=np.float32) < p).astype(np.float32)
    return _symmetrize(A)


def sherrington_kirkpatrick(n: int = 8192, seed: int = 1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    J = rng.standard_normal((n, n), dtype=np.float32)
    J = np.triu(J, 1)
    J = J + J.T
    J /= np.float32(np.sqrt(n))
    np.fill_diagonal(J, 0.0)
    return np.ascontiguousarray(J, dtype=np.float32)


def gnp_weighted(n: int, p: float, seed: int = 1, dist: str = "uniform") -> np.ndarray:
    rng = np.random.default_rng(seed)
    mask = rng.random((n, n), dtype=np.float32) < p
    if dist == "uniform":
        w = 1.0 - rng.random((n, n), dtype=np.float32)  # (0, 1]
    elif dist == "normal":
        w = rng.standard_normal((n, n), dtype=np.float32)
    else:
        raise ValueError(dist)
    return _symmetrize(np.where(mask, w, np.float32(0.0)))


def batched_uneven(count: int = 512, lo: int = 64, hi: int = 1024, seed: int = 7):
    """Instances of the batched workload: n ~ U[lo, hi]; even slots 3-regular +-1,
    odd slots G(n, 0.1) with uniform (0, 1] weights."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(lo, hi + 1, size=count)
    out = []
    for i, n in enumerate(sizes):
        n = int(n)
        if i % 2 == 0:
            if n % 2:  # a 3-regular graph needs an even node count
                n += 1 if n < hi else -1
            out.append(regular_pm1_fast(n, seed=int(rng.integers(1 << 30))))
        else:
            out.append(gnp_weighted(n, 0.1, seed=int(rng.integers(1 << 30)), dist="uniform"))
    return out


def regular_pm1_fast(n: int, seed: int, degree: int = 3) -> np.ndarray:
    """3-regular +-1 instance via networkx with a numpy-drawn sign per edge."""
    import networkx as nx

    G = nx.random_regular_graph(d=degree, n=n, seed=seed)
    rng = np.random.default_rng(seed)
    W = np.zeros((n, n), dtype=np.float32)
    e = np.array(list(G.edges()), dtype=np.int64)
    s = rng.choice(np.array([-1.0, 1.0], dtype=np.float32), size=len(e))
    W[e[:, 0], e[:, 1]] = s
    W[e[:, 1], e[:, 0]] = s
    return W


def random_bits(n: int, seed: int, batch: int | None = None) -> np.ndarray:
    rng = np.random.default_rng(seed)
    shape = (n,) if batch is None else (batch, n)
    return rng.random(shape) < 0.5


def regular_pm1_np(n: int, seed: int, degree: int = 3, max_tries: int = 1000) -> np.ndarray:
    """Random `degree`-regular graph with a +-1 weight per edge, drawn with the
    pairing model in numpy (shuffle n * degree stubs, pair neighbours, retry
    while a pair is a loop or repeats an edge): uniform over simple regular
    graphs, and fast enough to stream thousands of training graphs."""
    if (n * degree) % 2:
        raise ValueError("n * degree must be even")
    rng = np.random.default_rng(seed)
    stubs = np.repeat(np.arange(n, dtype=np.int64), degree)
    for _ in range(max_tries):
        rng.shuffle(stubs)
        a, b = stubs[0::2], stubs[1::2]
        if np.any(a == b):
            continue
        lo, hi = np.minimum(a, b), np.maximum(a, b)
        key = lo * n + hi
        if np.unique(key).size != key.size:
            continue
        W = np.zeros((n, n), dtype=np.float32)
        s = rng.choice(np.array([-1.0, 1.0], dtype=np.float32), size=key.size)
        W[lo, hi] = s
        W[hi, lo] = s
        return W
    raise RuntimeError("no simple regular graph drawn")


def proposal_training_graph(i: int, seed: int = 0, lo: int = 128, hi: int = 2048) -> np.ndarray:
    """The i-th graph of the proposal-network training stream: n ~ U[lo, hi];
    even i: 3-regular +-1, odd i: G(n, 0.05) with N(0, 1) weights."""
    rng = np.random.default_rng([seed, i])
    n = int(rng.integers(lo, hi + 1))
    s = int(rng.integers(1 << 30))
    if i % 2 == 0:
        return regular_pm1_np(n + (n % 2), seed=s)
    return gnp_weighted(n, 0.05, seed=s, dist="normal")
