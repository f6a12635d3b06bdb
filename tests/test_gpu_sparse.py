"""Sparse-input entry points on the GPU against the reference's sparse path
(golden_sparse.npz) and against the dense entry points on the same graph."""

import importlib
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "golden_sparse.npz")


def test_sampler_init_reads_the_stored_rows():
    from scipy.sparse import csr_matrix

    import torch
    from pyqrackising_b200.device import DeviceGraph
    from pyqrackising_b200.sparse import sparse_to_dense

    MT = importlib.import_module("pyqrackising_b200.maxcut_tfim")
    z = np.load(GOLD)
    for i in range(int(z["count"])):
        _, W, S = sparse_to_dense(csr_matrix(z[f"U{i}"]))
        dg = DeviceGraph(W)
        J, deg, _ = MT.hamming_cdf(dg, 2, 8.0, 8.0, jz_W=torch.from_numpy(S).cuda())
        np.testing.assert_allclose(J.cpu().numpy(), z[f"J{i}"], rtol=1e-12, atol=1e-12)
        assert np.array_equal(deg.cpu().numpy(), z[f"deg{i}"])


def test_exhaustive_below_the_sparse_threshold():
    from scipy.sparse import csr_matrix

    from pyqrackising_b200 import maxcut_tfim_sparse

    z = np.load(GOLD)
    checked = 0
    for i in range(int(z["count"])):
        if f"exact{i}_0_val" not in z:
            continue
        G = csr_matrix(z[f"U{i}"])
        for spin in (0, 1):
            bits, val, _ = maxcut_tfim_sparse(G, is_spin_glass=bool(spin))
            ref_val = float(z[f"exact{i}_{spin}_val"])
            if ref_val < 0.0:
                assert bits == "0" * G.shape[0] and val == 0.0
            else:
                sol = "".join("1" if b else "0" for b in z[f"exact{i}_{spin}_sol"])
                assert bits == sol and val == pytest.approx(ref_val, rel=1e-6, abs=1e-6)
            checked += 1
    assert checked >= 2


def test_sparse_solver_equals_dense_solver_from_the_same_start(oracle_mod):
    from scipy.sparse import csr_matrix

    from pyqrackising_b200 import spin_glass_solver, spin_glass_solver_sparse

    O = oracle_mod
    z = np.load(GOLD)
    for i in (0, 1):
        U = z[f"U{i}"]
        W = U + U.T
        guess = [bool(b) for b in z[f"states{i}"][0]]
        for spin in (True, False):
            a = spin_glass_solver_sparse(csr_matrix(U), best_guess=guess, is_spin_glass=spin)
            b = spin_glass_solver(W, best_guess=guess, is_spin_glass=spin)
            assert a[0] == b[0] and a[1] == b[1] and a[3] == b[3]
            bits = np.array([c == "1" for c in a[0]])
            assert a[1] == pytest.approx(O.compute_cut(bits, W), rel=1e-9, abs=1e-6)


def test_sampling_path_returns_a_rescored_cut(oracle_mod):
    from scipy.sparse import csr_matrix

    from pyqrackising_b200 import maxcut_tfim_sparse

    O = oracle_mod
    MT = importlib.import_module("pyqrackising_b200.maxcut_tfim")
    z = np.load(GOLD)
    U = z["U1"]
    MT.set_seed(3)
    bits, val, (l, r) = maxcut_tfim_sparse(csr_matrix(U), quality=2)
    sol = np.array([c == "1" for c in bits])
    assert val == pytest.approx(O.compute_cut(sol, U + U.T), rel=1e-6, abs=1e-6)
    assert len(l) + len(r) == U.shape[0]


def test_device_expansion_equals_the_host_expansion():
    """pqi_coo_to_dense builds W and S bit for bit as the host does, for graph
    and matrix inputs and both triangles stored; repeated coordinates take the
    host path; an out-of-range coordinate is reported, not written."""
    import ctypes

    import networkx as nx
    import torch
    from scipy.sparse import coo_matrix, csr_matrix

    from pyqrackising_b200 import _lib
    from pyqrackising_b200 import device as D
    from pyqrackising_b200.sparse import sparse_to_dense, sparse_to_device

    z = np.load(GOLD)
    rng = np.random.default_rng(3)
    cases = []
    for i in range(int(z["count"])):
        U = z[f"U{i}"]
        cases += [csr_matrix(U), csr_matrix(U + U.T)]
        g = nx.Graph()
        g.add_nodes_from(range(U.shape[0]))
        for a, b in zip(*np.nonzero(U)):
            g.add_edge(int(b), int(a), weight=float(U[a, b]))
        cases.append(g)
    n = 300
    r, c = rng.integers(0, n, 4000), rng.integers(0, n, 4000)
    cases.append(csr_matrix((rng.standard_normal(4000).astype(np.float32), (r, c)), shape=(n, n)))
    cases.append(coo_matrix((rng.standard_normal(4000).astype(np.float32), (r, c)), shape=(n, n)))
    for G in cases:
        _, W, S = sparse_to_dense(G)
        _, Wd, Sd = sparse_to_device(G)
        assert np.array_equal(Wd.cpu().numpy().view(np.uint32), W.view(np.uint32))
        assert np.array_equal(Sd.cpu().numpy().view(np.uint32), S.view(np.uint32))
    rows = torch.tensor([0, 5, 1], dtype=torch.int32, device="cuda")
    cols = torch.tensor([1, 0, 2], dtype=torch.int32, device="cuda")
    vals = torch.tensor([1.0, 2.0, 3.0], dtype=torch.float32, device="cuda")
    W = torch.empty((3, 3), dtype=torch.float32, device="cuda")
    bad = torch.empty(1, dtype=torch.int32, device="cuda")
    _lib.call("pqi_coo_to_dense", D._ptr(rows), D._ptr(cols), D._ptr(vals), ctypes.c_longlong(3), 3,
              None, D._ptr(W), D._ptr(bad), D.stream_ptr())
    assert int(bad.item()) == 1
    assert W.cpu().numpy().tolist() == [[0.0, 1.0, 0.0], [1.0, 0.0, 3.0], [0.0, 3.0, 0.0]]


def test_graph_without_stored_entries():
    """A 30-node sparse matrix with no stored entries: the device expansion
    gives zero matrices and the solver returns a zero cut."""
    from scipy.sparse import csr_matrix

    from pyqrackising_b200 import spin_glass_solver_sparse
    from pyqrackising_b200.sparse import sparse_to_device

    G = csr_matrix((30, 30), dtype=np.float32)
    _, W, S = sparse_to_device(G)
    assert float(W.abs().sum()) == 0.0 and float(S.abs().sum()) == 0.0
    bits, cut, (l, r), energy = spin_glass_solver_sparse(G, best_guess="0" * 30)
    assert len(bits) == 30 and cut == 0.0 and energy == 0.0 and len(l) + len(r) == 30


def test_hybrid_is_the_dense_seed_then_the_sparse_solver():
    """spin_glass_solver_hybrid (spin_glass_solver_hybrid.py:7-46): with the
    sampler's seed fixed it returns what the two steps return run by hand;
    anything but an nx.Graph is refused, as in the reference."""
    import importlib

    import networkx as nx

    from pyqrackising_b200 import spin_glass_solver_hybrid, spin_glass_solver_sparse

    MT = importlib.import_module("pyqrackising_b200.maxcut_tfim")
    rng = np.random.default_rng(9)
    g = nx.random_regular_graph(3, 40, seed=4)
    for u, v in g.edges():
        g[u][v]["weight"] = float(rng.choice([-1.0, 1.0]))
    for spin in (True, False):
        MT.set_seed(5)
        got = spin_glass_solver_hybrid(g, quality=2, is_spin_glass=spin)
        MT.set_seed(5)
        guess, _, _ = MT.maxcut_tfim(g, quality=2, is_spin_glass=spin)
        want = spin_glass_solver_sparse(g, best_guess=guess, is_spin_glass=spin)
        MT.set_seed(None)
        assert got == want
    with pytest.raises(TypeError):
        spin_glass_solver_hybrid(np.zeros((30, 30), dtype=np.float32))
