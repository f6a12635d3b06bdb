"""Travelling-salesman drop-in: ``tsp_symmetric`` and ``tsp_asymmetric``
(pyqrackising/tsp.py:559-1162), the recursive bipartition heuristic that
calls the MAXCUT solver on its subgraphs.

A tour of n >= 7 cities is split into two halves, each half is toured
recursively (brute force below 7 cities), the halves are joined
(``stitch_*``), the joined path is re-split and re-joined (``restitch``), and
the top level is polished with 2-opt and a neighbour-restricted 3-opt. The
split is either a random partition (``monte_carlo=True``, the reference's
default) or a maximum cut of the subgraph (``monte_carlo=False``).

The MAXCUT splits run on the device. With ``split="batched"`` (the default
for ``monte_carlo=False``) the recursion is split level by level: every
subgraph of one recursion depth is cut in the same ``BatchedSolver`` launch
(steepest ascent from ``32 * multi_start`` random starts per subgraph plus
kicked rounds, best cut per subgraph), so a tour costs one device launch per
depth instead of one solver call per subgraph. ``split="solver"`` calls the
``spin_glass_solver`` drop-in once per subgraph with the caller's
quality/shots/anneal arguments, as the reference does (tsp.py:657-672).

The path heuristics are compiled CPU code (numba), step for step the
reference's, so that a run with the same random stream returns the same tour:
the candidate lengths are full left-to-right path sums compared with strict
'<' (2-opt: tsp.py:27-162; 3-opt: :165-301), the joins and re-splits draw
their random numbers in the reference's order (:419-455), and the brute force
keeps the reference's edge sums (:456-556, including the cyclic search that
leaves out the last edge before the closing one). ``seed(s)`` seeds that
stream (numba's generator, the one the reference's compiled helpers draw
from). ``is_parallel=True`` selects the chunked 2-opt/3-opt variants (chunks
of ``os.cpu_count()`` candidates, evaluated against the same path, then
accepted in order) and runs both halves in this process.
"""

from __future__ import annotations

import itertools
import os

import numpy as np
from numba import njit

_CHUNK = os.cpu_count() or 1


@njit(cache=True)
def seed(s):
    """Seed the random stream of the compiled helpers (splits and re-splits)."""
    np.random.seed(s)


# ---------------------------------------------------------------------------
# Path lengths and 2-opt (tsp.py:17-162)


@njit(cache=True)
def path_length(path, G):
    total = 0.0
    for t in range(path.shape[0] - 1):
        total += G[path[t], path[t + 1]]
    return total


@njit(cache=True)
def _reversed_length(best, G, i, j):
    """Length of `best` with best[i:j] reversed (i >= 1), summed left to right
    as path_length sums the rebuilt path."""
    total = 0.0
    prev = best[0]
    for t in range(1, best.shape[0]):
        cur = best[i + j - 1 - t] if (t >= i and t < j) else best[t]
        total += G[prev, cur]
        prev = cur
    return total


@njit(cache=True)
def _reverse_copy(p, i, j):
    out = p.copy()
    for t in range(i, j):
        out[t] = p[i + j - 1 - t]
    return out


@njit(cache=True)
def _two_opt(path, G, i0, i_off, j_off, chunk):
    """Segment reversals p[i:j] for i in [i0, L - i_off), j in [i + 2,
    L - j_off), first improvement kept and the scan continued on the new
    path; chunk > 0: j in chunks of `chunk`, each chunk's candidates from the
    path at the chunk's start, then accepted in order when below the best."""
    best = path.copy()
    best_d = path_length(best, G)
    L = best.shape[0]
    improved = True
    while improved:
        improved = False
        for i in range(i0, L - i_off):
            if chunk <= 0:
                for j in range(i + 2, L - j_off):
                    d = _reversed_length(best, G, i, j)
                    if d < best_d:
                        best = _reverse_copy(best, i, j)
                        best_d = d
                        improved = True
            else:
                for j in range(i + 2, L - j_off, chunk):
                    m = min(chunk, L - j_off - j)
                    snap = best
                    ds = np.empty(m)
                    for k in range(m):
                        ds[k] = _reversed_length(snap, G, i, j + k)
                    for k in range(m):
                        if ds[k] < best_d:
                            best = _reverse_copy(snap, i, j + k)
                            best_d = ds[k]
                            improved = True
    return best, best_d


def one_way_two_opt(path, G, parallel=False):
    return _two_opt(np.asarray(path, dtype=np.int64), G, 1, 1, 0, _CHUNK if parallel else 0)


def anchored_two_opt(path, G, parallel=False):
    return _two_opt(np.asarray(path, dtype=np.int64), G, 2, 1, 0, _CHUNK if parallel else 0)


def two_opt(path, G, parallel=False):
    return _two_opt(np.asarray(path, dtype=np.int64), G, 1, 2, 1, _CHUNK if parallel else 0)


# ---------------------------------------------------------------------------
# Neighbour-restricted 3-opt (tsp.py:165-301)


@njit(cache=True)
def _three_opt_move(P, i, j, k, case):
    A = P[: i + 1]
    B = P[i + 1 : j + 1]
    C = P[j + 1 : k + 1]
    D = P[k + 1 :]
    if case == 0:
        return np.concatenate((A, B[::-1], C, D))
    if case == 1:
        return np.concatenate((A, B, C[::-1], D))
    if case == 2:
        return np.concatenate((A, B[::-1], C[::-1], D))
    if case == 3:
        return np.concatenate((A, C, B, D))
    if case == 4:
        return np.concatenate((A, C[::-1], B[::-1], D))
    if case == 5:
        return np.concatenate((A, C, B[::-1], D))
    return np.concatenate((A, C[::-1], B, D))


@njit(cache=True)
def _three_opt(path, W, nbr, chunked):
    """Positions i < j < k with j from the neighbour list of the node at i and
    k from that of the node at position j (the reference indexes positions
    by neighbour node ids), the seven reconnections in the reference's
    order; the first improvement restarts the scan (chunked: all seven from
    the same path, then accepted in order)."""
    n = path.shape[0]
    best = path.copy()
    best_d = path_length(best, W)
    improved = True
    while improved:
        improved = False
        cur = best
        for i in range(n - 5):
            for jj in range(nbr.shape[1]):
                j = nbr[cur[i], jj]
                if j <= i or j >= n - 3:
                    continue
                for kk in range(nbr.shape[1]):
                    k = nbr[cur[j], kk]
                    if k <= j or k >= n - 1:
                        continue
                    if chunked:
                        snap = best
                        ds = np.empty(7)
                        for case in range(7):
                            ds[case] = path_length(_three_opt_move(snap, i, j, k, case), W)
                        for case in range(7):
                            if ds[case] < best_d:
                                best = _three_opt_move(snap, i, j, k, case)
                                best_d = ds[case]
                                improved = True
                    else:
                        for case in range(7):
                            cand = _three_opt_move(best, i, j, k, case)
                            d = path_length(cand, W)
                            if d < best_d:
                                best = cand
                                best_d = d
                                improved = True
                                break
                    if improved:
                        break
                if improved:
                    break
            if improved:
                break
    return best, best_d


def targeted_three_opt(path, W, neighbor_lists, parallel=False):
    return _three_opt(np.asarray(path, dtype=np.int64), W, neighbor_lists, parallel)


def neighbor_lists(G_m, k):
    """Per node, the k nodes of smallest weight G_m[i, j] (itself included),
    ascending, ties by the lower node; entries of weight +inf or NaN never
    count, and short lists are padded with node 0 (tsp.py:802-814)."""
    n = G_m.shape[0]
    out = np.zeros((n, k), dtype=np.int64)
    for i in range(n):
        row = G_m[i]
        ok = np.nonzero(row < np.inf)[0]
        order = ok[np.argsort(row[ok], kind="stable")][:k]
        out[i, : len(order)] = order
    return out


# ---------------------------------------------------------------------------
# Joins and re-splits (tsp.py:324-433)


@njit(cache=True)
def _insert(p, i, q):
    return np.concatenate((p[:i], q, p[i:]))


@njit(cache=True)
def stitch_singlet(G, s, bulk):
    best_w = G[s, bulk[0]]
    w = G[s, bulk[-1]]
    single = np.array([s], dtype=np.int64)
    if w < best_w:
        best_w = w
        best = np.concatenate((bulk, single))
    else:
        best = np.concatenate((single, bulk))
    for i in range(1, bulk.shape[0]):
        w = G[s, bulk[i - 1]] + G[s, bulk[i]] - G[bulk[i - 1], bulk[i]]
        if w < best_w:
            best_w = w
            best = _insert(bulk, i, single)
    return best


@njit(cache=True)
def stitch(G, path_a, path_b, symmetric):
    """Join two paths: end to end (either order), or one inserted into an
    edge of the other, in either orientation, both ways round. Symmetric:
    the cheapest connection. Asymmetric: the connection weighed with both
    paths' lengths in their current orientation, reset per orientation (the
    reference keeps its end-to-end choice as the bound, tsp.py:381-416)."""
    if path_a.shape[0] == 1:
        return stitch_singlet(G, path_a[0], path_b)
    if path_b.shape[0] == 1:
        return stitch_singlet(G, path_b[0], path_a)
    a, b = path_a, path_b
    best_connect = G[a[-1], b[0]]
    w = G[a[0], b[-1]]
    if w < best_connect:
        best_connect = w
        best = np.concatenate((b, a))
    else:
        best = np.concatenate((a, b))
    for _outer in range(2):
        for _inner in range(2):
            ta0, ta1 = a[0], a[-1]
            if symmetric:
                for i in range(1, b.shape[0]):
                    w = G[ta0, b[i - 1]] + G[ta1, b[i]] - G[b[i - 1], b[i]]
                    if w < best_connect:
                        best_connect = w
                        best = _insert(b, i, a)
            else:
                pw = path_length(a, G) + path_length(b, G)
                best_w = best_connect + pw
                for i in range(1, b.shape[0]):
                    w = G[ta0, b[i - 1]] + G[ta1, b[i]] - G[b[i - 1], b[i]]
                    if (w + pw) < best_w:
                        best_w = w + pw
                        best = _insert(b, i, a)
            a = a[::-1].copy()
        a, b = b, a
    return best


@njit(cache=True)
def restitch(G, path, symmetric):
    l = path.shape[0]
    mid = ((l + 1) if (l & 1) and (np.random.random() < 0.5) else l) >> 1
    if mid < 4:
        return path
    pa = restitch(G, path[:mid].copy(), symmetric)
    pb = restitch(G, path[mid:].copy(), symmetric)
    return stitch(G, pa, pb, symmetric)


@njit(cache=True)
def monte_carlo_split(n):
    """A random partition with both sides non-empty: one draw per node, side a
    below 0.5, redrawn whole until neither side is empty (tsp.py:436-455)."""
    while True:
        a = np.empty(n, dtype=np.int64)
        b = np.empty(n, dtype=np.int64)
        na = 0
        nb = 0
        for i in range(n):
            if np.random.random() < 0.5:
                a[na] = i
                na += 1
            else:
                b[nb] = i
                nb += 1
        if na > 0 and nb > 0:
            return a[:na].copy(), b[:nb].copy()


@njit(cache=True)
def sub_matrix(G, idx):
    m = idx.shape[0]
    out = np.zeros((m, m), dtype=np.float64)
    for i in range(m):
        for j in range(m):
            if i != j:
                out[i, j] = G[idx[i], idx[j]]
    return out


# ---------------------------------------------------------------------------
# Brute force (tsp.py:456-556, 845-858)


def _brute_force(G_m, n, cyclic):
    """First permutation of least weight, sums in the reference's order."""
    if cyclic:
        perms = np.array(list(itertools.permutations(range(1, n))), dtype=np.int64)
        full = np.hstack((np.zeros((len(perms), 1), dtype=np.int64), perms))
        w = np.zeros(len(perms))
        for t in range(perms.shape[1] - 1):  # (the reference stops one edge short)
            w += G_m[full[:, t], full[:, t + 1]]
        w += G_m[full[:, -1], full[:, 0]]
    else:
        full = np.array(list(itertools.permutations(range(n))), dtype=np.int64)
        w = np.zeros(len(full))
        for t in range(n - 1):
            w += G_m[full[:, t], full[:, t + 1]]
    b = int(np.argmin(w))
    path = [int(x) for x in full[b]]
    if cyclic:
        path.append(path[0])
    return path, float(w[b])


def _small_symmetric(G_m, n, nodes, cyclic):
    # n <= 3: the reference keeps the heavier of the orientations (:523-556)
    if n == 3:
        if cyclic:
            w0 = G_m[0, 1] + G_m[1, 2] + G_m[2, 0]
            w1 = G_m[0, 2] + G_m[2, 1] + G_m[1, 0]
            if w0 >= w1:
                return nodes + [nodes[0]], float(w0)
            r = nodes[::-1]
            return [r[2]] + r, float(w1)
        w012 = G_m[0, 1] + G_m[1, 2]
        w021 = G_m[0, 1] + G_m[0, 2]
        w120 = G_m[0, 2] + G_m[1, 2]
        if w012 >= w021 and w012 >= w120:
            return nodes, float(w012)
        if w021 >= w012 and w021 >= w120:
            return [nodes[1], nodes[0], nodes[2]], float(w021)
        return [nodes[0], nodes[2], nodes[1]], float(w120)
    if n == 2:
        if cyclic:
            return nodes + [nodes[0]], float(2 * G_m[0, 1])
        return nodes, float(G_m[0, 1])
    return nodes, 0


def _small_asymmetric(G_m, n, nodes, cyclic):
    if n == 2:
        w = G_m[0, 1]
        if G_m[1, 0] < w:
            w = G_m[1, 0]
            nodes = nodes[::-1]
        if cyclic:
            return nodes + [nodes[0]], float(2 * w)
        return nodes, float(w)
    return nodes, 0


# ---------------------------------------------------------------------------
# MAXCUT splits on the device


def _cut_sides(bits, n):
    a = [i for i in range(n) if not bits[i]]
    b = [i for i in range(n) if bits[i]]
    return a, b


def _solver_split(G_cut, opts):
    """The reference's loop (tsp.py:656-672): spin_glass_solver until both
    sides are non-empty, best cut over multi_start runs."""
    from .spin_glass_solver import spin_glass_solver

    best_cut, a, b = -float("inf"), [], []
    for _ in range(opts["multi_start"]):
        sides = ([], [])
        while len(sides[0]) == 0 or len(sides[1]) == 0:
            _, cut_value, sides, _ = spin_glass_solver(
                G_cut, is_spin_glass=False, quality=opts["quality"], shots=opts["shots"],
                anneal_t=opts["anneal_t"], anneal_h=opts["anneal_h"], repulsion_base=opts["repulsion_base"])
        if cut_value > best_cut:
            best_cut = cut_value
            a, b = list(sides[0]), list(sides[1])
    return a, b


def _batched_splits(mats, opts):
    """Maximum cuts of several subgraphs in one batched launch: best of
    32 * multi_start random starts per subgraph (steepest ascent, then kicked
    rounds); a subgraph whose best cut leaves a side empty falls back to the
    solver loop."""
    from .batch import BatchedSolver
    from .device import DeviceGraph

    graphs = [DeviceGraph(np.ascontiguousarray(m, dtype=np.float32)) for m in mats]
    solver = BatchedSolver(graphs, 32 * max(1, int(opts["multi_start"])), False, rounds=4,
                           kick=max(1, min(8, min(g.n for g in graphs) // 4)), seed=int(opts["seed"]))
    solver.set_starts(int(opts["seed"]))
    solver.step()
    _, states, _, _ = solver.results()
    out = []
    for g, m in enumerate(mats):
        n = m.shape[0]
        words = states[g].cpu().numpy().view(np.uint32)
        bits = np.unpackbits(words.view(np.uint8), bitorder="little")[:n].astype(bool)
        a, b = _cut_sides(bits, n)
        if not a or not b:
            a, b = _solver_split(m, opts)
        out.append((a, b))
    return out


# ---------------------------------------------------------------------------
# The recursion (tsp.py:559-843 symmetric, 845-1162 asymmetric)


def _header(G_m, nodes, n, start_node, end_node, cyclic, symmetric, split):
    """(a, b, c, is_reversed, G_sub) of one recursion node (tsp.py:628-683,
    944-1002). A cyclic tour ignores start and end nodes; an end node alone
    acts as the start (asymmetric: on G^T, the result reversed). `split`
    gives the partition when no start node anchors it. The sub-matrices come
    from G_sub (G^T when reversed); everything after the recursion uses the
    caller's G and the caller's start and end nodes, as the reference's
    drivers do."""
    reversed_ = False
    G_sub = G_m
    if cyclic:
        start_node = None
        end_node = None
    if start_node is None and end_node is not None:
        if not symmetric:
            reversed_ = True
            G_sub = G_m.T
        start_node = end_node
        end_node = None
    c = []
    if start_node is None:
        a, b = split()
    else:
        a = [nodes.index(start_node)]
        b = [i for i in range(n) if i != a[0]]
        if end_node is not None:
            c = [nodes.index(end_node)]
            b.remove(c[0])
    return a, b, c, reversed_, G_sub


class _Splits:
    """Partitions of the recursion nodes, keyed by their position in the
    recursion (a string of 'a'/'b' steps): precomputed level by level for the
    batched MAXCUT splits, drawn on demand otherwise."""

    def __init__(self, mode, opts):
        self.mode, self.opts, self.table = mode, opts, {}

    def get(self, key, G_cut, n):
        if self.mode == "random":
            a, b = monte_carlo_split(n)
            return [int(x) for x in a], [int(x) for x in b]
        if self.mode == "solver":
            return _solver_split(G_cut, self.opts)
        return self.table[key]


def _plan_batched(G_m, nodes, n, start_node, end_node, cyclic, symmetric, opts):
    """Every split of a monte_carlo=False recursion, one batched launch per
    depth: the partitions depend only on each subgraph, and the children of a
    node are its two sub-matrices."""
    table = {}
    level = []
    if n >= 7:
        if cyclic or (start_node is None and end_node is None):
            level.append(("", G_m))
        else:
            # an anchored root is split by its start (and end) node, not cut
            a, b, _, _, G_sub = _header(G_m, nodes, n, start_node, end_node, cyclic, symmetric, None)
            for tag, side in (("a", a), ("b", b)):
                if len(side) >= 7:
                    level.append((tag, sub_matrix(G_sub, np.asarray(side, dtype=np.int64))))
    while level:
        mats = [(m + m.T) / 2 if not symmetric else m for _, m in level]
        cuts = _batched_splits(mats, opts)
        nxt = []
        for (key, m), (a, b) in zip(level, cuts):
            table[key] = (a, b)
            for tag, side in (("a", a), ("b", b)):
                if len(side) >= 7:
                    nxt.append((key + tag, sub_matrix(m, np.asarray(side, dtype=np.int64))))
        level = nxt
    return table


def _tsp(G_m, nodes, n, start_node, end_node, cyclic, top, k_neighbors, symmetric, parallel, splits, key):
    if n < 7:
        if n > (3 if symmetric else 2):
            path, w = _brute_force(G_m, n, cyclic)
            return [nodes[x] for x in path], w
        return (_small_symmetric if symmetric else _small_asymmetric)(G_m, n, list(nodes), cyclic)

    G_cut = G_m if symmetric else (G_m + G_m.T) / 2
    a, b, c, reversed_, G_sub = _header(G_m, nodes, n, start_node, end_node, cyclic, symmetric,
                                        lambda: splits.get(key, G_cut, n))
    ia, ib = np.asarray(a, dtype=np.int64), np.asarray(b, dtype=np.int64)
    G_a, G_b = sub_matrix(G_sub, ia), sub_matrix(G_sub, ib)
    sol_a = _tsp(G_a, list(range(len(a))), len(a), None, None, False, False, 0, symmetric, parallel, splits, key + "a")
    sol_b = _tsp(G_b, list(range(len(b))), len(b), None, None, False, False, 0, symmetric, parallel, splits, key + "b")
    nbr = neighbor_lists(G_m, k_neighbors) if k_neighbors > 0 else np.zeros((1, 1), dtype=np.int64)
    path_a = ia[np.asarray(sol_a[0], dtype=np.int64)]
    path_b = ib[np.asarray(sol_b[0], dtype=np.int64)]
    if start_node is None:
        best = stitch(G_m, path_a, path_b, symmetric)
    elif symmetric:
        # (the reference compares both ends of b against a's first node)
        best = np.concatenate((path_a, path_b))
        if G_m[path_a[0], path_b[-1]] < G_m[path_a[0], path_b[0]]:
            best = np.concatenate((path_a, path_b[::-1]))
    else:
        best = np.concatenate((path_a, path_b))
    if c:
        best = np.concatenate((best, np.asarray(c, dtype=np.int64)))
    best = restitch(G_m, best, symmetric)
    if top:
        best = _polish(G_m, best, cyclic, start_node, end_node, k_neighbors, nbr, symmetric, parallel)
    w = path_length(best, G_m)
    if reversed_:
        best = best[::-1]
    return [nodes[int(x)] for x in best], w


def _polish(G_m, best, cyclic, start_node, end_node, k_neighbors, nbr, symmetric, parallel):
    """The top level's 2-opt variant and 3-opt (tsp.py:592-623); asymmetric:
    each pass also on the reversed path, the shorter kept (:881-929)."""
    if cyclic:
        best = np.concatenate((best, best[:1]))
        first = two_opt
    elif end_node is not None:
        first = two_opt
    elif start_node is not None:
        first = anchored_two_opt
    else:
        first = one_way_two_opt
    if symmetric:
        best, _ = first(best, G_m, parallel)
        if k_neighbors > 0:
            best, _ = targeted_three_opt(best, G_m, nbr, parallel)
        return best
    path, w = first(best.copy(), G_m, parallel)
    # (reversed: plain two_opt where start_node anchors the forward pass)
    second = two_opt if first is anchored_two_opt else first
    rpath, rw = second(best[::-1].copy(), G_m, parallel)
    if rw < w:
        path, w = rpath, rw
    if k_neighbors > 0:
        best = path
        path, w = targeted_three_opt(best.copy(), G_m, nbr, parallel)
        rpath, rw = targeted_three_opt(best[::-1].copy(), G_m, nbr, parallel)
        if rw < w:
            path, w = rpath, rw
    return path


def _entry(G, start_node, end_node, quality, shots, anneal_t, anneal_h, repulsion_base, monte_carlo,
           k_neighbors, is_cyclic, multi_start, is_top_level, is_parallel, symmetric, split, split_seed):
    from .util import as_matrix

    nodes, G_m = as_matrix(G)
    G_m = np.asarray(G_m)
    n = len(nodes)
    opts = {"quality": quality, "shots": shots, "anneal_t": anneal_t, "anneal_h": anneal_h,
            "repulsion_base": repulsion_base, "multi_start": int(multi_start), "seed": split_seed}
    if monte_carlo:
        splits = _Splits("random", opts)
    elif split == "solver":
        splits = _Splits("solver", opts)
    elif split == "batched":
        splits = _Splits("batched", opts)
        splits.table = _plan_batched(G_m, nodes, n, start_node, end_node, is_cyclic, symmetric, opts)
    else:
        raise ValueError("split must be 'batched' or 'solver'")
    return _tsp(G_m, nodes, n, start_node, end_node, bool(is_cyclic), bool(is_top_level), int(k_neighbors),
                symmetric, bool(is_parallel), splits, "")


def tsp_symmetric(G, start_node=None, end_node=None, quality=None, shots=None, anneal_t=None, anneal_h=None,
                  repulsion_base=None, monte_carlo=True, k_neighbors=20, is_cyclic=True, multi_start=1,
                  is_top_level=True, is_parallel=False, parallel_level=0, *, split="batched", split_seed=0):
    """(tour as node labels, weight) of a symmetric instance (an nx.Graph or a
    dense matrix), the reference's tsp_symmetric (tsp.py:686-842). A cyclic
    tour repeats its first node at the end. split / split_seed: the MAXCUT
    splits of monte_carlo=False (module docstring)."""
    del parallel_level  # (the halves run in this process)
    return _entry(G, start_node, end_node, quality, shots, anneal_t, anneal_h, repulsion_base, monte_carlo,
                  k_neighbors, is_cyclic, multi_start, is_top_level, is_parallel, True, split, split_seed)


def tsp_asymmetric(G, start_node=None, end_node=None, quality=None, shots=None, anneal_t=None, anneal_h=None,
                   repulsion_base=None, monte_carlo=True, k_neighbors=20, is_cyclic=True, multi_start=1,
                   is_top_level=True, is_parallel=False, parallel_level=0, *, split="batched", split_seed=0):
    """The reference's tsp_asymmetric (tsp.py:1005-1162): splits on the
    symmetrised weights (G + G^T) / 2, paths weighed on G itself; an end node
    without a start node runs on G^T and reverses the result."""
    del parallel_level
    return _entry(G, start_node, end_node, quality, shots, anneal_t, anneal_h, repulsion_base, monte_carlo,
                  k_neighbors, is_cyclic, multi_start, is_top_level, is_parallel, False, split, split_seed)
