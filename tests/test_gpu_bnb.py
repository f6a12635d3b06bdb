"""The exact branch-and-bound solver on the GPU (pqi_bnb_eval behind
solve_maxcut_bnb) against the reference's own results
(tests/golden/golden_bnb.npz) and the oracle (oracle/bnb_oracle.py)."""

import ctypes
import itertools
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "golden_bnb.npz")


def _cases():
    z = np.load(GOLD)
    return z, [str(s) for s in z["names"]]


def test_same_results_as_the_reference_with_its_batch_cap():
    from pyqrackising_b200 import solve_maxcut_bnb

    z, names = _cases()
    cap = int(z["batch_cap"])
    for name in names:
        W = z[f"{name}_W"]
        spin = bool(z[f"{name}_spin"])
        bits, cut, (l, r), energy, certified = solve_maxcut_bnb(
            W, best_guess=str(z[f"{name}_guess"]), is_spin_glass=spin, verbose=False, batch_size=cap)
        assert bits == str(z[f"{name}_bits"]), name
        assert cut == pytest.approx(float(z[f"{name}_cut"]), rel=1e-6, abs=1e-6), name
        assert energy == pytest.approx(float(z[f"{name}_energy"]), rel=1e-6, abs=1e-6), name
        assert certified is True and len(l) + len(r) == W.shape[0]


def test_other_batch_sizes_follow_the_oracle():
    """Batch sizes 1 and 4096 visit nodes in other orders: the states and
    values equal the oracle's with the same batch size; for MAXCUT the
    certified cut is the reference's. (For spin glasses the reference bounds
    energies with the cut bound, so its result depends on the order.)"""
    from oracle import bnb_oracle as B
    from pyqrackising_b200 import solve_maxcut_bnb

    z, names = _cases()
    for name in names:
        W = z[f"{name}_W"]
        spin = bool(z[f"{name}_spin"])
        guess = str(z[f"{name}_guess"])
        for cap in (1, 4096):
            bits, cut, _, energy, certified = solve_maxcut_bnb(
                W, best_guess=guess, is_spin_glass=spin, verbose=False, batch_size=cap)
            obits, ocut, oenergy, _ = B.solve(W, guess, spin, cap)
            assert certified and bits == obits, (name, cap)
            assert cut == pytest.approx(ocut, rel=1e-6, abs=1e-6)
            assert energy == pytest.approx(oenergy, rel=1e-6, abs=1e-6)
            if not spin:
                assert cut == pytest.approx(float(z[f"{name}_cut"]), rel=1e-6, abs=1e-6)


def test_node_evaluation_matches_the_oracle():
    """Bounds (float64, bit for bit), pruning, leaf values and branch variables
    of random partial assignments, float and integer weights."""
    from oracle import bnb_oracle as B
    from pyqrackising_b200 import _lib
    from pyqrackising_b200 import device as D

    rng = np.random.default_rng(5)
    for kind in ("normal", "int"):
        n = 20
        if kind == "normal":
            U = np.where(rng.random((n, n)) < 0.4, rng.standard_normal((n, n)), 0.0)
        else:
            U = rng.choice([-2.0, -1.0, 0.0, 1.0, 3.0], size=(n, n))
        U = np.triu(U, 1).astype(np.float32)
        W = (U + U.T).astype(np.float32)
        count = 700
        fv = rng.integers(-1, 2, size=(count, n)).astype(np.int8)
        fv[: count // 3] = np.where(fv[: count // 3] < 0, 1, fv[: count // 3])  # leaves
        ubs = np.array([B.upper_bound(W, row) for row in fv])
        best = float(np.median(ubs))
        Wd = torch.from_numpy(W).cuda()
        fvd = torch.from_numpy(np.ascontiguousarray(fv.T)).cuda()
        ub = torch.empty(count, dtype=torch.float64, device="cuda")
        leaf = torch.empty(count, dtype=torch.float64, device="cuda")
        br = torch.empty(count, dtype=torch.int32, device="cuda")
        st = torch.empty(count, dtype=torch.int8, device="cuda")
        for spin in (0, 1):
            _lib.call("pqi_bnb_eval", D._ptr(Wd), n, D._ptr(fvd), count, ctypes.c_double(best), spin,
                      D._ptr(ub), D._ptr(leaf), D._ptr(br), D._ptr(st), D.stream_ptr())
            assert np.array_equal(ub.cpu().numpy(), ubs)
            s, lv, bv = st.cpu().numpy(), leaf.cpu().numpy(), br.cpu().numpy()
            for b in range(count):
                if ubs[b] <= best + 1e-9:
                    assert s[b] == 0
                elif np.all(fv[b] >= 0):
                    assert s[b] == 1
                    assert lv[b] == (B.leaf_energy(W, fv[b]) if spin else B.leaf_cut(W, fv[b]))
                else:
                    assert s[b] == 2 and bv[b] == int(np.argmax(B.influence_scores(W, fv[b])))


def test_heuristic_warm_start_and_time_limit():
    from oracle import bnb_oracle as B
    from pyqrackising_b200 import solve_maxcut_bnb

    z, _ = _cases()
    W = z["reg16_cut_W"]
    n = W.shape[0]
    best = max(B.objectives(W, np.array(bits, dtype=bool))[0] for bits in itertools.product([0, 1], repeat=n))
    bits, cut, _, _, certified = solve_maxcut_bnb(W, verbose=False)
    assert certified and cut == pytest.approx(best)
    _, _, _, _, certified = solve_maxcut_bnb(W, best_guess="0" * n, verbose=False, time_limit=-1.0)
    assert certified is False


def test_graph_input_and_tiny_graphs():
    """nx.Graph input (nodes in graph order, missing weights read as 1.0) and
    the reference's answers below three nodes (solve_maxcut_bnb.py:263-271)."""
    import networkx as nx

    from oracle import bnb_oracle as B
    from pyqrackising_b200 import solve_maxcut_bnb

    g = nx.Graph()
    labels = ["a", "b", "c", "d", "e", "f", "g"]
    g.add_nodes_from(labels)
    for u, v, w in [("a", "b", 2.0), ("b", "c", None), ("c", "d", -1.0), ("d", "a", 3.0), ("e", "f", 1.5),
                    ("f", "g", 2.5), ("g", "e", -0.5), ("a", "e", 1.0)]:
        if w is None:
            g.add_edge(u, v)
        else:
            g.add_edge(u, v, weight=w)
    W = nx.to_numpy_array(g, nodelist=labels, weight="weight", nonedge=0.0, dtype=np.float32)
    guess = "0101010"
    bits, cut, (l, r), energy, certified = solve_maxcut_bnb(g, best_guess=guess, verbose=False, batch_size=4)
    obits, ocut, oen, _ = B.solve(W, guess, False, 4)
    assert certified and bits == obits and cut == pytest.approx(ocut) and energy == pytest.approx(oen)
    assert sorted(l + r) == sorted(labels) and all(labels[i] in r for i, ch in enumerate(bits) if ch == "1")
    assert solve_maxcut_bnb(np.zeros((0, 0), dtype=np.float32), verbose=False) == ("", 0, ([], []), 0, True)
    assert solve_maxcut_bnb(np.zeros((1, 1), dtype=np.float32), verbose=False) == ("0", 0, ([0], []), 0, True)
    pos = np.array([[0.0, 2.0], [2.0, 0.0]], dtype=np.float32)
    assert solve_maxcut_bnb(pos, verbose=False) == ("01", 2.0, ([0], [1]), -2.0, True)
    neg = -pos
    assert solve_maxcut_bnb(neg, verbose=False) == ("00", 0, ([0, 1], []), -2.0, True)


def test_sparse_input_matches_the_reference_sparse_solver():
    """solve_maxcut_bnb_sparse on the upper-triangular CSR of each fixture
    graph (and on the same graph as nx input) returns the reference sparse
    solver's bit strings, values and certificates."""
    import networkx as nx
    from scipy.sparse import csr_matrix

    from pyqrackising_b200 import solve_maxcut_bnb_sparse

    z, names = _cases()
    cap = int(z["batch_cap"])
    for name in names:
        W = z[f"{name}_W"]
        spin = bool(z[f"{name}_spin"])
        guess = str(z[f"{name}_guess"])
        g = nx.Graph()
        g.add_nodes_from(range(W.shape[0]))
        for a, b in zip(*np.nonzero(np.triu(W, 1))):
            g.add_edge(int(a), int(b), weight=float(W[a, b]))
        for G in (csr_matrix(np.triu(W, 1)), g):
            bits, cut, _, energy, certified = solve_maxcut_bnb_sparse(
                G, best_guess=guess, is_spin_glass=spin, verbose=False, batch_size=cap)
            assert bits == str(z[f"{name}_sparse_bits"]), name
            assert cut == pytest.approx(float(z[f"{name}_sparse_cut"]), rel=1e-6, abs=1e-6), name
            assert energy == pytest.approx(float(z[f"{name}_sparse_energy"]), rel=1e-6, abs=1e-6), name
            assert certified == bool(z[f"{name}_sparse_certified"])
