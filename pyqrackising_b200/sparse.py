"""Sparse-input entry points: spin_glass_solver_sparse and maxcut_tfim_sparse
(pyqrackising/spin_glass_solver_sparse.py:517-864,
pyqrackising/maxcut_tfim_sparse.py:373-472), same signatures and returns.

The reference's sparse kernels sum every stored CSR entry (u, v) once
(kernels.cl:233-251), which is the dense form with
W = G_offdiag + G_offdiag^T: a graph's sparse and dense objectives, flip
values and pair values agree, and only the summation order differs. On a B200
the graph is therefore expanded to that dense matrix in HBM (n = 65536 takes
17 GB of 180), where the tensor-core scoring and the row-streaming flip kernels
run. Only the coordinate list crosses to the device (12 bytes per stored
entry); pqi_coo_to_dense scatters it into W and into S, the matrix of the
stored entries alone. What the sparse path does differently is
kept: the exhaustive search below n = 23 (maxcut_tfim_util.py:166) and the
sampler's J_eff and degrees read from the stored (upper-triangular) rows
(maxcut_tfim_sparse.py:204-224). Diagonal entries (self-loops) are dropped:
they change no cut.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from . import device as D
from .maxcut_tfim import _maxcut_tfim
from .spin_glass_solver import _spin_glass_solver

HEURISTIC_THRESHOLD_SPARSE = 23  # maxcut_tfim_util.py:166


def sparse_coordinates(G):
    """(nodes, n, rows, cols, vals, unique) of the stored off-diagonal entries:
    an nx.Graph is read as the reference reads it (upper triangle in node order,
    weight default 1.0, maxcut_tfim_util.py:533-542); a scipy sparse matrix is
    used as given. `unique` is False when a coordinate repeats (a non-canonical
    scipy matrix or a multigraph); those entries are summed on the host."""
    try:
        import networkx as nx
    except ImportError:  # pragma: no cover
        nx = None
    is_graph = nx is not None and isinstance(G, nx.Graph)
    if is_graph:
        nodes = list(G.nodes())
        n = len(nodes)
        index = {u: i for i, u in enumerate(nodes)}
        m = G.number_of_edges()
        rows = np.empty(m, dtype=np.int64)
        cols = np.empty(m, dtype=np.int64)
        vals = np.empty(m, dtype=np.float32)
        for e, (u, v, w) in enumerate(G.edges(data="weight", default=1.0)):
            rows[e], cols[e], vals[e] = index[u], index[v], w
        rows, cols = np.minimum(rows, cols), np.maximum(rows, cols)
    else:
        coo = G.tocoo()
        n = coo.shape[0]
        nodes = list(range(n))
        rows, cols = coo.row.astype(np.int64), coo.col.astype(np.int64)
        vals = coo.data.astype(np.float32)
    keep = rows != cols
    rows, cols, vals = rows[keep], cols[keep], vals[keep]
    if is_graph:
        unique = not isinstance(G, nx.MultiGraph)
    else:
        unique = bool(getattr(G, "has_canonical_format", False))
    if not unique:
        unique = np.unique(rows * n + cols).size == rows.size
    return nodes, n, rows, cols, vals, unique


def sparse_to_device(G, device=None):
    """(nodes, W, S) as sparse_to_dense, with W and S built on the device from
    the coordinate list (torch float32 n x n). Falls back to the host
    expansion, then one upload, when coordinates repeat (the host sums them in
    the reference's order)."""
    dev = torch.device(device) if device is not None else D.default_device()
    nodes, n, rows, cols, vals, unique = sparse_coordinates(G)
    if not unique:
        nodes, W, S = sparse_to_dense(G)
        return nodes, torch.from_numpy(W).to(dev), torch.from_numpy(S).to(dev)
    r = torch.from_numpy(rows.astype(np.int32)).to(dev)
    c = torch.from_numpy(cols.astype(np.int32)).to(dev)
    v = torch.from_numpy(vals).to(dev)
    W = torch.empty((n, n), dtype=torch.float32, device=dev)
    S = torch.empty((n, n), dtype=torch.float32, device=dev)
    bad = torch.empty(1, dtype=torch.int32, device=dev)
    _lib.call(
        "pqi_coo_to_dense",
        D._ptr(r),
        D._ptr(c),
        D._ptr(v),
        ctypes.c_longlong(int(rows.size)),
        int(n),
        D._ptr(S),
        D._ptr(W),
        D._ptr(bad),
        D.stream_ptr(),
    )
    if int(bad.item()):
        raise ValueError("sparse matrix has a coordinate outside its shape")
    return nodes, W, S


def _dense_operands(G):
    """Host matrices below the exhaustive-search size (those runs use host
    arrays), device matrices from there on."""
    n = G.number_of_nodes() if hasattr(G, "number_of_nodes") else G.shape[0]
    if n < HEURISTIC_THRESHOLD_SPARSE:
        return sparse_to_dense(G)
    return sparse_to_device(G)


def sparse_to_dense(G):
    """(nodes, dense symmetric W, stored-rows matrix S) from an nx.Graph (read
    as the reference does: upper triangle in node order, weight default 1.0,
    maxcut_tfim_util.py:533-542) or a scipy sparse matrix (used as given).
    S holds the stored entries off the diagonal (the rows the sampler's J and
    degrees are read from); W = S + S^T."""
    try:
        import networkx as nx
    except ImportError:  # pragma: no cover
        nx = None
    if nx is not None and isinstance(G, nx.Graph):
        nodes = list(G.nodes())
        n = len(nodes)
        index = {u: i for i, u in enumerate(nodes)}
        S = np.zeros((n, n), dtype=np.float32)
        for u, v, d in G.edges(data=True):
            i, j = index[u], index[v]
            if i == j:
                continue
            a, b = (i, j) if i < j else (j, i)
            S[a, b] = np.float32(d.get("weight", 1.0))
    else:
        coo = G.tocoo()
        n = coo.shape[0]
        nodes = list(range(n))
        S = np.zeros((n, n), dtype=np.float32)
        keep = coo.row != coo.col
        np.add.at(S, (coo.row[keep], coo.col[keep]), coo.data[keep].astype(np.float32))
    W = S + S.T
    return nodes, W, S


def maxcut_tfim_sparse(
    G,
    quality=None,
    shots=None,
    is_spin_glass=False,
    anneal_t=None,
    anneal_h=None,
    repulsion_base=None,
    is_maxcut_gpu=True,
    is_nested=False,
):
    nodes, W, S = _dense_operands(G)
    return _maxcut_tfim(nodes, W, quality, shots, is_spin_glass, anneal_t, anneal_h, repulsion_base,
                        threshold=HEURISTIC_THRESHOLD_SPARSE, jz_matrix=S)


def spin_glass_solver_sparse(
    G,
    quality=None,
    shots=None,
    best_guess=None,
    is_maxcut_gpu=True,
    is_spin_glass=True,
    anneal_t=None,
    anneal_h=None,
    repulsion_base=None,
    is_log=False,
    gray_iterations=None,
    gray_seed_multiple=None,
    bp_scale=None,
    bp_damping=0.5,
):
    nodes, W, S = _dense_operands(G)
    return _spin_glass_solver(nodes, W, quality, shots, best_guess, is_maxcut_gpu, is_spin_glass, anneal_t,
                              anneal_h, repulsion_base, gray_iterations, gray_seed_multiple, bp_scale, bp_damping,
                              threshold=HEURISTIC_THRESHOLD_SPARSE, jz_matrix=S)


def spin_glass_solver_hybrid(
    G,
    quality=None,
    shots=None,
    is_maxcut_gpu=True,
    is_spin_glass=True,
    anneal_t=None,
    anneal_h=None,
    repulsion_base=None,
    is_log=False,
    gray_iterations=None,
    gray_seed_multiple=None,
    bp_scale=None,
    bp_damping=0.5,
):
    """The dense maxcut_tfim seed followed by the sparse solver from that seed
    (pyqrackising/spin_glass_solver_hybrid.py:7-46); G must be an nx.Graph."""
    import networkx as nx

    from .maxcut_tfim import maxcut_tfim

    if not isinstance(G, nx.Graph):
        raise TypeError("G graph must be a networkx.Graph for maxcut_hybrid!")
    guess, _, _ = maxcut_tfim(G, quality=quality, shots=shots, repulsion_base=repulsion_base,
                              is_maxcut_gpu=is_maxcut_gpu, is_spin_glass=is_spin_glass, anneal_t=anneal_t,
                              anneal_h=anneal_h)
    return spin_glass_solver_sparse(G, best_guess=guess, is_maxcut_gpu=is_maxcut_gpu, is_spin_glass=is_spin_glass,
                                    is_log=is_log, gray_iterations=gray_iterations,
                                    gray_seed_multiple=gray_seed_multiple, bp_scale=bp_scale, bp_damping=bp_damping)
