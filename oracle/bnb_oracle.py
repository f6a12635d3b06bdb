"""TEST INFRASTRUCTURE ONLY: a plain-Python restatement of the reference's exact
branch-and-bound solver (pyqrackising/solve_maxcut_bnb.py), the checker for
pyqrackising_b200.solve_maxcut_bnb.

Only ``tests/`` may import this module; the product never does. Every sum runs
in the reference's order in float64 over float32 weights, so bounds, leaf values
and branching scores equal the reference's, and with the same batch cap the
traversal (and so the returned state) is the reference's. Pinned against
``tests/golden/golden_bnb.npz`` (results of the reference itself). Small n only.
"""

from __future__ import annotations

import numpy as np


def upper_bound(W, row):
    """_upper_bound_batch for one node (solve_maxcut_bnb.py:47-71)."""
    n = W.shape[0]
    total = 0.0
    for i in range(n):
        fi = row[i]
        for j in range(i + 1, n):
            w = W[i, j]
            if w == 0.0:
                continue
            fj = row[j]
            if fi >= 0 and fj >= 0:
                if fi != fj:
                    total += float(w)
            elif w > 0.0:
                total += float(w)
    return total


def leaf_cut(W, row):
    """_eval_leaves_cut for one node (solve_maxcut_bnb.py:74-84)."""
    n = W.shape[0]
    cut = 0.0
    for i in range(n):
        for j in range(i + 1, n):
            if W[i, j] != 0.0 and row[i] != row[j]:
                cut += float(W[i, j])
    return cut


def leaf_energy(W, row):
    """_eval_leaves_energy for one node (solve_maxcut_bnb.py:87-97)."""
    n = W.shape[0]
    energy = 0.0
    for i in range(n):
        for j in range(i + 1, n):
            val = float(W[i, j])
            energy += -val if row[i] == row[j] else val
    return energy


def influence_scores(W, row):
    """_influence_scores (solve_maxcut_bnb.py:100-121)."""
    n = W.shape[0]
    scores = np.full(n, -1.0)
    for i in range(n):
        if row[i] >= 0:
            continue
        s = 0.0
        for j in range(n):
            if i == j or row[j] >= 0:
                continue
            s += float(abs(W[min(i, j), max(i, j)]))
        scores[i] = s
    return scores


def branch_and_bound(W, warm_theta, warm_energy, is_spin_glass, batch_cap):
    """_branch_and_bound (solve_maxcut_bnb.py:128-199) without printing or a time
    limit. Returns (best bits, best value, nodes explored, nodes pruned)."""
    W = np.asarray(W, dtype=np.float32)
    n = W.shape[0]
    best_bits = np.asarray(warm_theta, dtype=np.bool_).copy()
    best_value = float(warm_energy)
    stack = [np.full(n, -1, dtype=np.int8)]
    explored = pruned = 0
    while stack:
        size = min(batch_cap, len(stack))
        batch = [stack.pop() for _ in range(size)]
        explored += size
        ubs = [upper_bound(W, row) for row in batch]
        leaves, interior = [], []
        for k in range(size):
            if ubs[k] <= best_value + 1e-9:
                pruned += 1
                continue
            if int(np.sum(batch[k] < 0)) == 0:
                leaves.append(k)
            else:
                interior.append(k)
        if leaves:
            vals = [leaf_energy(W, batch[k]) if is_spin_glass else leaf_cut(W, batch[k]) for k in leaves]
            b = int(np.argmax(vals))
            if vals[b] > best_value:
                best_value = float(vals[b])
                best_bits = (batch[leaves[b]] >= 1).copy()
        for k in interior:
            row = batch[k]
            var = int(np.argmax(influence_scores(W, row)))
            warm_val = int(best_bits[var])
            for val in (warm_val, 1 - warm_val):
                child = row.copy()
                child[var] = np.int8(val)
                stack.append(child)
    return best_bits, best_value, explored, pruned


def objectives(W, bits):
    """(cut, energy) of a state in float64 (maxcut_tfim_util.py:319-331)."""
    W = np.asarray(W, dtype=np.float64)
    x = np.where(np.asarray(bits, dtype=np.bool_), 1.0, -1.0)
    total = np.triu(W, 1).sum()
    q = x @ np.triu(W, 1) @ x
    return (total - q) / 2.0, -q


def solve(W, guess, is_spin_glass, batch_cap):
    """solve_maxcut_bnb (solve_maxcut_bnb.py:208-321) from a given best_guess
    bit string: (bit string, cut, energy, certified)."""
    W = np.asarray(W, dtype=np.float32)
    theta = np.array([c == "1" for c in guess], dtype=np.bool_)
    cut0, en0 = objectives(W, theta)
    warm = en0 if is_spin_glass else cut0
    bits, value, _, _ = branch_and_bound(W, theta, warm, is_spin_glass, batch_cap)
    cut, en = objectives(W, bits)
    bitstring = "".join("1" if b else "0" for b in bits)
    if is_spin_glass:
        return bitstring, cut, -value, True
    return bitstring, value, en, True
