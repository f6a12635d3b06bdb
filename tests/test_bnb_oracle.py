"""The branch-and-bound oracle (oracle/bnb_oracle.py) against the reference's
own results (tests/golden/golden_bnb.npz, made by
tests/golden/make_bnb_golden.py) and against exhaustive search."""

import itertools
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden", "golden_bnb.npz")


def _cases():
    z = np.load(GOLD)
    return z, [str(s) for s in z["names"]]


def test_oracle_reproduces_the_reference_results():
    from oracle import bnb_oracle as B

    z, names = _cases()
    cap = int(z["batch_cap"])
    for name in names:
        W = z[f"{name}_W"]
        spin = bool(z[f"{name}_spin"])
        bits, cut, energy, certified = B.solve(W, str(z[f"{name}_guess"]), spin, cap)
        assert bits == str(z[f"{name}_bits"]), name
        assert cut == pytest.approx(float(z[f"{name}_cut"]), rel=1e-6, abs=1e-6), name
        assert energy == pytest.approx(float(z[f"{name}_energy"]), rel=1e-6, abs=1e-6), name
        assert certified == bool(z[f"{name}_certified"])


def test_oracle_maxcut_value_is_the_exhaustive_optimum():
    from oracle import bnb_oracle as B

    z, names = _cases()
    for name in names:
        W = z[f"{name}_W"]
        if bool(z[f"{name}_spin"]) or W.shape[0] > 14:
            continue
        n = W.shape[0]
        best = max(B.objectives(W, np.array(bits, dtype=bool))[0]
                   for bits in itertools.product([0, 1], repeat=n))
        _, cut, _, _ = B.solve(W, str(z[f"{name}_guess"]), False, int(z["batch_cap"]))
        assert cut == pytest.approx(best, rel=1e-6, abs=1e-6), name


def test_host_loop_follows_the_oracle_with_a_cpu_evaluator(monkeypatch):
    """The product's B&B host loop (stack, pops, pushes, incumbent) driven by a
    CPU stand-in for the device evaluation (the oracle's per-node bound, leaf
    and score): same final state and value as the oracle's loop for several
    batch sizes, on every fixture case."""
    import importlib

    from oracle import bnb_oracle as B

    M = importlib.import_module("pyqrackising_b200.solve_maxcut_bnb")

    class CpuEvaluator:
        def __init__(self, W, cap):
            self.W = W

        def __call__(self, batch, best_value, is_spin_glass):
            count = batch.shape[0]
            state = np.zeros(count, dtype=np.int8)
            leaf = np.zeros(count)
            branch = np.zeros(count, dtype=np.int32)
            for b in range(count):
                if B.upper_bound(self.W, batch[b]) <= best_value + 1e-9:
                    continue
                if np.all(batch[b] >= 0):
                    state[b] = 1
                    leaf[b] = B.leaf_energy(self.W, batch[b]) if is_spin_glass else B.leaf_cut(self.W, batch[b])
                else:
                    state[b] = 2
                    branch[b] = int(np.argmax(B.influence_scores(self.W, batch[b])))
            return state, leaf, branch

    monkeypatch.setattr(M, "_Evaluator", CpuEvaluator)
    z, names = _cases()
    for name in names:
        W = z[f"{name}_W"]
        if W.shape[0] > 14:
            continue
        spin = bool(z[f"{name}_spin"])
        theta = np.array([c == "1" for c in str(z[f"{name}_guess"])])
        cut0, en0 = B.objectives(W, theta)
        warm = en0 if spin else cut0
        for cap in (1, 7, 64):
            bits, value, certified = M._branch_and_bound(W, theta, warm, W.shape[0], spin, verbose=False,
                                                         batch_size=cap)
            obits, ovalue, _, _ = B.branch_and_bound(W, theta, warm, spin, cap)
            assert certified and np.array_equal(bits, obits) and value == ovalue, (name, cap)
