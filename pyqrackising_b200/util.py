"""Host helpers with the reference's conventions (pyqrackising/maxcut_tfim_util.py).

These are bookkeeping on the host (string building, argument parsing); all
arithmetic on the coupling matrix runs on the GPU through libpqi.
"""

from __future__ import annotations

import numpy as np

HEURISTIC_THRESHOLD = 24  # maxcut_tfim_util.py:165
GRAY_NODE_LIMIT = 131072  # maxcut_tfim_util.py:11 (kept for reference; no limit here)


def int_to_bitstring(integer: int, length: int) -> str:
    """LSB-first bit string of `integer` (maxcut_tfim_util.py:510-511)."""
    return (bin(integer)[2:].zfill(length))[::-1]


def parse_best_guess(best_guess, n: int):
    """best_guess as str / int (LSB = node 0, bool included) / list -> bool[n],
    anything else -> None (spin_glass_solver.py:484-491)."""
    if isinstance(best_guess, str):
        bitstring = best_guess
    elif isinstance(best_guess, int):
        bitstring = int_to_bitstring(best_guess, n)
    elif isinstance(best_guess, list):
        bitstring = "".join(["1" if b else "0" for b in best_guess])
    else:
        return None
    return np.array([b == "1" for b in bitstring], dtype=np.bool_)


def get_cut(solution, nodes):
    """(bit string, left nodes, right nodes) (maxcut_tfim_util.py:482-494)."""
    sol = np.asarray(solution, dtype=np.bool_)
    bit_string = "".join("1" if b else "0" for b in sol)
    l = [nodes[i] for i in range(len(sol)) if not sol[i]]
    r = [nodes[i] for i in range(len(sol)) if sol[i]]
    return bit_string, l, r


def as_matrix(G, dtype=np.float32):
    """(nodes, dense float32 matrix) for an nx.Graph or an array-like, as the
    reference converts its input (spin_glass_solver.py:454-465)."""
    try:
        import networkx as nx
    except ImportError:  # pragma: no cover
        nx = None
    if nx is not None and isinstance(G, nx.Graph):
        nodes = list(G.nodes())
        return nodes, nx.to_numpy_array(G, weight="weight", nonedge=0.0, dtype=dtype)
    n = len(G)
    return list(range(n)), G
