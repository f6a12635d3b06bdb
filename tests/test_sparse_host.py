"""Sparse-input host logic on CPU: CSR / graph -> the dense form the device
path uses, against the reference's sparse objectives (golden_sparse.npz,
made by tests/golden/make_sparse_golden.py from the reference itself)."""

import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden", "golden_sparse.npz")


def _cases():
    z = np.load(GOLD)
    return z, int(z["count"])


def test_csr_and_graph_give_the_same_dense_form():
    import networkx as nx
    from scipy.sparse import csr_matrix

    from pyqrackising_b200.sparse import sparse_to_dense

    z, count = _cases()
    for i in range(count):
        U = z[f"U{i}"]
        nodes, W, S = sparse_to_dense(csr_matrix(U))
        assert np.array_equal(W, U + U.T) and np.array_equal(S, U)
        G = nx.Graph()
        G.add_nodes_from(range(U.shape[0]))
        for a, b in zip(*np.nonzero(U)):
            G.add_edge(int(a), int(b), weight=float(U[a, b]))
        nodes2, W2, S2 = sparse_to_dense(G)
        assert nodes2 == list(range(U.shape[0])) and np.array_equal(W2, W) and np.array_equal(S2, U)
    # both triangles stored: the reference sums every stored entry
    U = z["U0"]
    _, W3, _ = sparse_to_dense(csr_matrix(U + U.T))
    assert np.array_equal(W3, 2 * (U + U.T))


def test_dense_objectives_equal_reference_sparse_objectives(oracle_mod):
    from scipy.sparse import csr_matrix

    from pyqrackising_b200.sparse import sparse_to_dense

    O = oracle_mod
    z, count = _cases()
    for i in range(count):
        _, W, _ = sparse_to_dense(csr_matrix(z[f"U{i}"]))
        tol = 1e-5 * np.abs(W).sum()
        for s, c, e in zip(z[f"states{i}"], z[f"cut{i}"], z[f"energy{i}"]):
            assert O.compute_cut(s, W) == pytest.approx(c, abs=tol)
            assert O.compute_energy(s, W) == pytest.approx(e, abs=tol)


def test_coordinate_list_rebuilds_the_host_expansion():
    """The coordinate list that crosses to the device holds exactly the host
    expansion's stored entries (graph and matrix inputs; repeats flagged)."""
    import networkx as nx
    from scipy.sparse import coo_matrix, csr_matrix

    from pyqrackising_b200.sparse import sparse_coordinates, sparse_to_dense

    z, count = _cases()
    cases = []
    for i in range(count):
        U = z[f"U{i}"]
        cases.append(csr_matrix(U))
        cases.append(csr_matrix(U + U.T))  # both halves stored
        g = nx.Graph()
        g.add_nodes_from(range(U.shape[0]))
        for a, b in zip(*np.nonzero(U)):
            g.add_edge(int(b), int(a), weight=float(U[a, b]))  # reversed endpoints
        cases.append(g)
    for G in cases:
        nodes, n, rows, cols, vals, unique = sparse_coordinates(G)
        assert unique
        _, W, S = sparse_to_dense(G)
        S2 = np.zeros((n, n), dtype=np.float32)
        S2[rows, cols] = vals
        assert np.array_equal(S2, S) and np.array_equal(S2 + S2.T, W)
    dup = coo_matrix((np.array([1.0, 2.0, 3.0], dtype=np.float32), (np.array([0, 0, 1]), np.array([1, 1, 2]))),
                     shape=(3, 3))
    assert not sparse_coordinates(dup)[5]


def test_hybrid_refuses_matrix_input():
    """spin_glass_solver_hybrid takes an nx.Graph only, as the reference
    (spin_glass_solver_hybrid.py:22-23); the check runs before any device work."""
    from pyqrackising_b200 import spin_glass_solver_hybrid

    with pytest.raises(TypeError):
        spin_glass_solver_hybrid(np.zeros((30, 30), dtype=np.float32))
