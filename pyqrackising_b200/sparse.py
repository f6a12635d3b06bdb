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

Graphs whose dense form would not fit (``use_compressed_rows``) run on
compressed rows instead (``SparseDeviceGraph``, the ``pqi_csr_*`` kernels):
O(n + nnz) memory, O(degree) per flip, the same values and selections, and
the same sampler (its neighbour lists are the rows). Above 131072 nodes the
Gray stage is skipped, as in the reference's GPU branch.
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


class SparseDeviceGraph:
    """A sparse coupling matrix on one GPU in compressed rows (both triangles,
    columns ascending; ``pqi_csr``): O(n + nnz) device memory, so graphs too
    large for an n x n matrix fit (G(200000, 1e-4) is 48 MB here, 160 GB
    dense). The same methods as ``device.DeviceGraph`` that the search loop
    uses, with the same values and selections; a flip costs O(degree).
    W = S + S^T of the stored off-diagonal entries S, as the reference's sparse
    kernels read them (kernels.cl:233-251). The rows are built on the host
    (scipy, O(nnz)) and uploaded once: ptr int64, col int32, val float32."""

    def __init__(self, G, device=None, stream=None):
        import scipy.sparse as sp

        _lib.load()
        self.device = torch.device(device) if device is not None else D.default_device()
        self.stream = stream
        nodes, n, rows, cols, vals, _ = sparse_coordinates(G)
        if not np.all(np.isfinite(vals)):
            raise ValueError("coupling matrix has non-finite entries")
        self.nodes = nodes
        self.n = n
        U = sp.coo_matrix((vals, (rows, cols)), shape=(n, n), dtype=np.float32)
        self._stored = U.tocsr()  # the stored rows S (the sampler's J_eff and degrees)
        self._stored.sum_duplicates()
        self._stored.sort_indices()
        self._stored_dev = None
        Wsym = (U + U.T).tocsr()
        Wsym.sum_duplicates()
        Wsym.eliminate_zeros()
        Wsym.sort_indices()
        self.nnz = int(Wsym.nnz)
        self.ptr = torch.from_numpy(Wsym.indptr.astype(np.int64)).to(self.device)
        self.col = torch.from_numpy(Wsym.indices.astype(np.int32) if self.nnz else np.zeros(1, np.int32)).to(self.device)
        self.val = torch.from_numpy(Wsym.data.astype(np.float32) if self.nnz else np.zeros(1, np.float32)).to(self.device)
        r = np.repeat(np.arange(n), np.diff(Wsym.indptr))
        upper = Wsym.indices > r
        self._upper_sum = float(np.asarray(Wsym.data, dtype=np.float64)[upper].sum())
        d = np.asarray(Wsym.data)
        self.is_integer = bool(np.all(d == np.rint(d)) and (d.size == 0 or np.abs(d).max() <= 127))
        self.max_degree = int(np.diff(Wsym.indptr).max()) if n else 0
        self.csr = _lib.PqiCsr()
        self.csr.ptr = self.ptr.data_ptr()
        self.csr.col = self.col.data_ptr()
        self.csr.val = self.val.data_ptr()
        self.csr.n = n
        self.csr.nnz = self.nnz
        self.csr.upper_sum = self._upper_sum
        self.ws = D.Workspace(self.device)
        self.n32 = (n + 31) >> 5
        self.n64 = (n + 63) >> 6

    @property
    def upper_sum(self) -> float:
        return self._upper_sum

    def row_lists(self):
        """The rows as the TFIM sampler's neighbour lists (ptr, col, val)."""
        return self.ptr, self.col, self.val

    def tfim_jz(self, J_eff: torch.Tensor, degrees: torch.Tensor):
        """The sampler's J_eff and degrees from the stored rows S with the
        reference's sparse-path arithmetic (pqi_csr_tfim_jz)."""
        S = self._stored
        if self._stored_dev is None:
            self._stored_dev = (
                torch.from_numpy(S.indptr.astype(np.int64)).to(self.device),
                torch.from_numpy(S.indices.astype(np.int32) if S.nnz else np.zeros(1, np.int32)).to(self.device),
                torch.from_numpy(S.data.astype(np.float32) if S.nnz else np.zeros(1, np.float32)).to(self.device),
            )
        # min over all of S: the stored values, and the zeros of every row
        # (the diagonal is never stored, so each row has at least one zero)
        gmin = float(min(0.0, float(S.data.min()) if S.nnz else 0.0))
        p, c, v = self._stored_dev
        _lib.call("pqi_csr_tfim_jz", D._ptr(p), D._ptr(c), D._ptr(v), self.n, ctypes.c_float(gmin),
                  D._ptr(J_eff), D._ptr(degrees), self.sp())

    def sp(self):
        return D.stream_ptr(self.stream)

    def wsp(self, nbytes: int = 0):
        # scratch: keys, one float32 copy of the gains, selection and pair state
        return self.ws.get(max(int(nbytes), 16 * self.n + (1 << 16)))

    def pack(self, bits) -> torch.Tensor:
        return D.pack_bits(bits, self.n, self.device, self.stream)

    def unpack(self, words: torch.Tensor, rows: int = 1, pitch: int | None = None) -> np.ndarray:
        return D.unpack_bits(words, self.n, rows, pitch, self.device, self.stream)

    def gains(self, words: torch.Tensor, rows: int = 1, fp64: bool = True):
        g32 = torch.empty(rows * self.n, dtype=torch.float32, device=self.device)
        g64 = torch.empty(rows * self.n, dtype=torch.float64, device=self.device) if fp64 else None
        _lib.call("pqi_csr_gains", ctypes.byref(self.csr), D._ptr(words), rows, D._ptr(g32), D._ptr(g64), self.sp())
        return g32, g64

    def single_bit_flips(self, words, is_spin_glass, G, L):
        be = torch.empty(1, dtype=torch.float32, device=self.device)
        bi = torch.empty(1, dtype=torch.int32, device=self.device)
        wsp, wsn = self.wsp()
        _lib.call("pqi_csr_single_bit_flips", ctypes.byref(self.csr), D._ptr(words), int(bool(is_spin_glass)), G, L,
                  D._ptr(be), D._ptr(bi), wsp, wsn, self.sp())
        return be, bi

    def double_bit_flips(self, words, g64, is_spin_glass, G, L, improving=False):
        """(best value, 64-bit pair index) of one double-flip pass. improving:
        the same answer whenever the best value is > 0, else some value <= 0
        (pqi_csr_improving_double_flip: at a single-flip local optimum only the
        adjacent pairs are scored)."""
        be = torch.empty(1, dtype=torch.float32, device=self.device)
        bi = torch.empty(1, dtype=torch.int64, device=self.device)
        wsp, wsn = self.wsp()
        fn = "pqi_csr_improving_double_flip" if improving else "pqi_csr_double_bit_flips"
        _lib.call(fn, ctypes.byref(self.csr), D._ptr(words), D._ptr(g64),
                  int(bool(is_spin_glass)), G, L, D._ptr(be), D._ptr(bi), wsp, wsn, self.sp())
        return be, bi

    def apply_flip(self, words, g64, k, l=-1):
        _lib.call("pqi_csr_apply_flip", ctypes.byref(self.csr), D._ptr(words), D._ptr(g64), int(k), int(l), self.sp())

    def single_descent(self, words, g64, is_spin_glass, G, L, max_flips, trace=None):
        esum = torch.zeros(1, dtype=torch.float64, device=self.device)
        flips = torch.zeros(1, dtype=torch.int32, device=self.device)
        wsp, wsn = self.wsp()
        rc = _lib.status("pqi_csr_single_descent", ctypes.byref(self.csr), D._ptr(words), D._ptr(g64),
                         int(bool(is_spin_glass)), G, L, int(max_flips), D._ptr(esum), D._ptr(flips), D._ptr(trace),
                         wsp, wsn, self.sp())
        if rc not in (_lib.PQI_OK, _lib.PQI_ETIMEOUT):
            raise _lib.PQIError(rc, "pqi_csr_single_descent")
        return esum, flips, rc

    def gray(self, words64, g64, is_spin_glass, iters_bound, seeds):
        tout = torch.empty(seeds * self.n64 * 2, dtype=torch.int32, device=self.device)
        eout = torch.empty(seeds, dtype=torch.float32, device=self.device)
        resident = min(int(seeds), 148 * 4)
        wsp, wsn = self.wsp(resident * self.n * 8 + (1 << 16))
        _lib.call("pqi_csr_gray", ctypes.byref(self.csr), D._ptr(words64), D._ptr(g64), int(bool(is_spin_glass)),
                  ctypes.c_longlong(int(iters_bound)), int(seeds), D._ptr(tout), D._ptr(eout), wsp, wsn, self.sp())
        return tout, eout

    def select(self, values: torch.Tensor, G: int, L: int):
        be = torch.empty(1, dtype=torch.float32, device=self.device)
        bi = torch.empty(1, dtype=torch.int32, device=self.device)
        wsp, wsn = self.wsp()
        _lib.call("pqi_select", D._ptr(values), values.numel(), G, L, D._ptr(be), D._ptr(bi), wsp, wsn, self.sp())
        return be, bi

    def rescore(self, words: torch.Tensor, rows: int = 1):
        cut = torch.empty(rows, dtype=torch.float64, device=self.device)
        en = torch.empty(rows, dtype=torch.float64, device=self.device)
        _lib.call("pqi_csr_rescore_fp64", ctypes.byref(self.csr), D._ptr(words), rows, D._ptr(cut), D._ptr(en),
                  self.sp())
        return cut, en

    def calculate_cut(self, words: torch.Tensor, shots: int, is_spin_glass: bool, G: int, L: int, energies=True):
        e = torch.empty(shots, dtype=torch.float32, device=self.device) if energies else None
        be = torch.empty(1, dtype=torch.float32, device=self.device)
        bi = torch.empty(1, dtype=torch.int32, device=self.device)
        wsp, wsn = self.wsp(4 * shots + 16 * self.n + (1 << 16))
        _lib.call("pqi_csr_calculate_cut", ctypes.byref(self.csr), D._ptr(words), int(shots), int(bool(is_spin_glass)),
                  G, L, D._ptr(e), D._ptr(be), D._ptr(bi), wsp, wsn, self.sp())
        return e, be, bi


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


CSR_MIN_NODES = 4096  # below this the dense form always fits and is the faster one
DENSE_BYTES_PER_ENTRY = 16  # W, its zero-diagonal copy, the bf16 split and the stored rows S


def use_compressed_rows(n: int) -> bool:
    """Whether the sparse entry points run on compressed rows
    (``SparseDeviceGraph``) rather than the dense expansion: when the dense
    matrices would take more than half of the device's free memory.
    PQI_SPARSE_PATH=csr or =dense forces one (for tests and comparisons)."""
    import os

    force = os.environ.get("PQI_SPARSE_PATH", "auto")
    if force in ("csr", "dense"):
        return force == "csr" and n >= 3
    if n < CSR_MIN_NODES:
        return False
    free, _ = torch.cuda.mem_get_info()
    return DENSE_BYTES_PER_ENTRY * n * n > free // 2


def _graph_size(G) -> int:
    return G.number_of_nodes() if hasattr(G, "number_of_nodes") else G.shape[0]


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
    if _graph_size(G) >= HEURISTIC_THRESHOLD_SPARSE and use_compressed_rows(_graph_size(G)):
        sg = SparseDeviceGraph(G)
        return _maxcut_tfim(sg.nodes, None, quality, shots, is_spin_glass, anneal_t, anneal_h, repulsion_base,
                            threshold=HEURISTIC_THRESHOLD_SPARSE, dg=sg)
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
    if _graph_size(G) >= HEURISTIC_THRESHOLD_SPARSE and use_compressed_rows(_graph_size(G)):
        sg = SparseDeviceGraph(G)
        return _spin_glass_solver(sg.nodes, None, quality, shots, best_guess, is_maxcut_gpu, is_spin_glass,
                                  anneal_t, anneal_h, repulsion_base, gray_iterations, gray_seed_multiple, bp_scale,
                                  bp_damping, threshold=HEURISTIC_THRESHOLD_SPARSE, graph=sg)
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
