"""Drop-in ``maxcut_tfim`` on the B200 path.

Same signature, defaults and return tuple as the reference
(``pyqrackising/maxcut_tfim.py:342-422``). Below the heuristic threshold
(n < 24) the exhaustive search runs on the GPU with the reference's value order
and tie rule (``pqi_exact_search``); above it the TFIM-inspired sampler draws
candidate batches that the tensor-core scoring kernel evaluates.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from . import device as D
from .util import HEURISTIC_THRESHOLD, as_matrix, get_cut


def exact_search(G_m, is_spin_glass: bool, device=None):
    """(bool[n], best value) of exact_maxcut / exact_spin_glass (maxcut_tfim.py:288-339)."""
    dev = torch.device(device) if device is not None else D.default_device()
    n = len(G_m)
    W = torch.from_numpy(np.ascontiguousarray(G_m, dtype=np.float32)).to(dev)
    val = torch.empty(1, dtype=torch.float64, device=dev)
    mask = torch.empty(1, dtype=torch.int32, device=dev)
    ws = torch.empty(4096, dtype=torch.uint8, device=dev)
    _lib.call(
        "pqi_exact_search",
        ctypes.c_void_p(W.data_ptr()),
        n,
        int(bool(is_spin_glass)),
        ctypes.c_void_p(val.data_ptr()),
        ctypes.c_void_p(mask.data_ptr()),
        ctypes.c_void_p(ws.data_ptr()),
        ctypes.c_size_t(ws.numel()),
        D.stream_ptr(),
    )
    m = int(mask.item())
    bits = np.array([(m >> i) & 1 for i in range(n)], dtype=np.bool_)
    return bits, float(val.item())


def maxcut_tfim(
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
    nodes, G_m = as_matrix(G)
    n_qubits = len(G_m)

    if n_qubits < HEURISTIC_THRESHOLD:
        best_solution, best_value = exact_search(G_m, is_spin_glass)
        bit_string, l, r = get_cut(best_solution, nodes)
        if best_value < 0.0:
            return "0" * n_qubits, 0.0, (nodes, [])
        return bit_string, best_value, (l, r)

    raise NotImplementedError("TFIM sampler not built yet")
