"""Drop-in ``maxcut_tfim`` on the B200 path.

Same signature, defaults and return tuple as the reference
(``pyqrackising/maxcut_tfim.py:342-422``). Below the heuristic threshold
(n < 24) the exhaustive search runs on the GPU with the reference's value order
and tie rule (``pqi_exact_search``); above it the TFIM-inspired sampler draws
candidate batches on the GPU (``pqi_tfim_*``) that the tensor-core scoring
kernel evaluates, round after round while the best value improves, as the
reference's GPU branch does (``sample_for_opencl``). ``is_maxcut_gpu`` is
accepted and ignored (no CPU path). The sampler's generator is counter-based
and seeded (``set_seed``; the reference's is unseeded), so results are
reproducible for a fixed seed.
"""

from __future__ import annotations

import ctypes
import math
import os

import numpy as np
import torch

from . import _lib
from . import device as D
from .util import HEURISTIC_THRESHOLD, as_matrix, get_cut


def _as_device_f32(M, dev):
    """A host array or a torch tensor as a contiguous float32 tensor on `dev`."""
    if isinstance(M, torch.Tensor):
        return M.detach().to(device=dev, dtype=torch.float32).contiguous()
    return torch.from_numpy(np.ascontiguousarray(M, dtype=np.float32)).to(dev)


def exact_search(G_m, is_spin_glass: bool, device=None):
    """(bool[n], best value) of exact_maxcut / exact_spin_glass (maxcut_tfim.py:288-339)."""
    dev = torch.device(device) if device is not None else D.default_device()
    n = len(G_m)
    W = _as_device_f32(G_m, dev)
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
    return _maxcut_tfim(nodes, G_m, quality, shots, is_spin_glass, anneal_t, anneal_h, repulsion_base)


def _maxcut_tfim(nodes, G_m, quality, shots, is_spin_glass, anneal_t, anneal_h, repulsion_base,
                 threshold=HEURISTIC_THRESHOLD, jz_matrix=None, dg=None):
    """maxcut_tfim on a dense symmetric matrix (host array or device tensor).
    `threshold` is the size below which the exhaustive search runs;
    `jz_matrix` (default G_m) is the matrix whose rows give the sampler's J_eff
    and degrees (the sparse entry point passes the upper triangle, as the
    reference's sparse path reads it); `dg` is G_m already prepared on the
    device (the solver shares its own; a compressed-row graph, with G_m None,
    from the sparse entry points)."""
    n_qubits = dg.n if dg is not None else len(G_m)

    if n_qubits < threshold:
        best_solution, best_value = exact_search(G_m, is_spin_glass)
        bit_string, l, r = get_cut(best_solution, nodes)
        if best_value < 0.0:
            return "0" * n_qubits, 0.0, (nodes, [])
        return bit_string, best_value, (l, r)

    if quality is None:
        quality = 6
    if shots is None:
        shots = n_qubits << quality
    if anneal_t is None:
        anneal_t = 8.0
    if anneal_h is None:
        anneal_h = 8.0
    if repulsion_base is None:
        repulsion_base = 5.0

    if dg is None:
        dg = D.DeviceGraph(G_m)
    jz = None
    if jz_matrix is not None:
        jz = _as_device_f32(jz_matrix, dg.device)
    best_solution, best_value = sample_and_score(
        dg, int(quality), int(shots), bool(is_spin_glass), float(anneal_t), float(anneal_h), float(repulsion_base),
        jz_W=jz,
    )
    bit_string, l, r = get_cut(best_solution, nodes)
    if best_value < 0.0:
        return "0" * n_qubits, 0.0, (nodes, [])
    return bit_string, best_value, (l, r)


_seed = None


def set_seed(seed: int | None):
    """Seed of the sampler's counter-based generator (None: a fresh random seed
    per process, like the reference's unseeded generator)."""
    global _seed
    _seed = None if seed is None else int(seed) & 0xFFFFFFFFFFFFFFFF


def _current_seed() -> int:
    global _seed
    if _seed is None:
        env = os.getenv("PYQRACKISING_B200_SEED")
        _seed = int(env) if env else int.from_bytes(os.urandom(8), "little")
    return _seed


def init_thresholds(n_qubits: int) -> np.ndarray:
    """Initial Hamming-weight weights (maxcut_tfim_util.py:558-575): binomial
    coefficients, normalised with exact integers on the host. For even n the
    reference never writes the middle entry of its np.empty array (its value
    is whatever memory held); here it is 0.0."""
    n_bias = n_qubits + 1
    thresholds = np.zeros(n_bias, dtype=np.float64)
    normalizer = 0
    for q in range(n_qubits >> 1):
        normalizer += math.comb(n_qubits, q) << 1
    if n_qubits & 1:
        normalizer += math.comb(n_qubits, n_qubits >> 1)
    p = 1
    for q in range(n_qubits >> 1):
        val = p / normalizer
        thresholds[q] = val
        thresholds[n_bias - (q + 1)] = val
        p = math.comb(n_qubits, q + 1)
    if n_qubits & 1:
        thresholds[n_qubits >> 1] = p / normalizer
    return thresholds


def hamming_cdf(dg: D.DeviceGraph, quality: int, anneal_t: float, anneal_h: float, jz_W=None):
    """(J_eff, degrees, cum_prob) on the device (init_J_and_z + maxcut_hamming_cdf);
    J_eff and degrees come from the rows of `jz_W` (n x n float32 on the
    device; the sparse path's stored rows, summed with its float32 rule),
    default the graph's own matrix."""
    n = dg.n
    dev = dg.device
    lib = _lib.load()
    J_eff = torch.empty(n, dtype=torch.float64, device=dev)
    degrees = torch.empty(n, dtype=torch.int32, device=dev)
    if hasattr(dg, "tfim_jz"):
        # a compressed-row graph: its stored rows, the sparse path's float32 rule
        dg.tfim_jz(J_eff, degrees)
    else:
        wsp, wsn = dg.wsp(1)
        # the sparse path passes its stored rows and the reference's float32 rule
        _lib.call("pqi_tfim_jz_f32" if jz_W is not None else "pqi_tfim_jz",
                  D._ptr(jz_W if jz_W is not None else dg.W), n, D._ptr(J_eff), D._ptr(degrees), wsp, wsn, dg.sp())
    thr = torch.from_numpy(init_thresholds(n)).to(dev)
    cum = torch.empty(max(n - 1, 1), dtype=torch.float64, device=dev)
    ws = dg.ws.get(lib.pqi_tfim_cdf_workspace_bytes(n, quality))
    _lib.call(
        "pqi_tfim_cdf",
        D._ptr(J_eff),
        D._ptr(degrees),
        n,
        int(quality),
        float(anneal_t),
        float(anneal_h),
        D._ptr(thr),
        D._ptr(cum),
        ws[0],
        ws[1],
        dg.sp(),
    )
    return J_eff, degrees, cum


ADJ_MAX_FILL = 0.25  # row lists pay off below this fraction of nonzero entries
ADJ_MAX_BYTES = 4 << 30


def row_lists(dg: D.DeviceGraph):
    """The nonzero entries of W's rows as device lists (ptr int64[n+1], col
    int32, val float32), built once per prepared graph; None when W is too
    dense for lists to beat the row scan."""
    if hasattr(dg, "row_lists"):
        return dg.row_lists()  # a compressed-row graph: its rows are the lists
    if getattr(dg, "_row_lists", False) is not False:
        return dg._row_lists
    n = dg.n
    count = torch.empty(n, dtype=torch.int64, device=dg.device)
    _lib.call("pqi_tfim_adj_count", D._ptr(dg.W), n, D._ptr(count), dg.sp())
    counts = count.cpu().numpy()
    nnz = int(counts.sum())
    lists = None
    if nnz <= ADJ_MAX_FILL * n * n and nnz * 8 <= ADJ_MAX_BYTES:
        ptr = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(counts, out=ptr[1:])
        ptr_d = torch.from_numpy(ptr).to(dg.device)
        col = torch.empty(max(nnz, 1), dtype=torch.int32, device=dg.device)
        val = torch.empty(max(nnz, 1), dtype=torch.float32, device=dg.device)
        _lib.call("pqi_tfim_adj_fill", D._ptr(dg.W), n, D._ptr(ptr_d), D._ptr(col), D._ptr(val), dg.sp())
        lists = (ptr_d, col, val)
    dg._row_lists = lists
    return lists


def sample_batch(dg: D.DeviceGraph, cum, shots: int, repulsion_base: float, seed: int, round_: int, out=None,
                 lists="auto"):
    """One round of shot_loop (maxcut_tfim.py:139-145) on the device: `shots`
    candidates as packed words [shots, ceil(n/32)]. Graphs with few nonzero
    weights per row use row lists for the repulsion updates (`lists`: "auto",
    or False for the row scan; both give the same draws)."""
    n = dg.n
    lib = _lib.load()
    if out is None:
        out = torch.empty(shots * dg.n32 + 1, dtype=torch.int32, device=dg.device)
        out[-1] = 0  # spare word (single-row 64-bit view), never written by the sampler
    ws = dg.ws.get(lib.pqi_tfim_sample_workspace_bytes(n))
    rl = row_lists(dg) if lists == "auto" else None
    if rl is not None:
        _lib.call(
            "pqi_tfim_sample_adj",
            D._ptr(getattr(dg, "W", None)),
            n,
            D._ptr(rl[0]),
            D._ptr(rl[1]),
            D._ptr(rl[2]),
            D._ptr(cum),
            float(repulsion_base),
            ctypes.c_uint64(seed),
            ctypes.c_uint64(round_),
            int(shots),
            D._ptr(out),
            ws[0],
            ws[1],
            dg.sp(),
        )
        return out
    _lib.call(
        "pqi_tfim_sample",
        D._ptr(dg.W),
        n,
        D._ptr(cum),
        float(repulsion_base),
        ctypes.c_uint64(seed),
        ctypes.c_uint64(round_),
        int(shots),
        D._ptr(out),
        ws[0],
        ws[1],
        dg.sp(),
    )
    return out


def sample_and_score(dg: D.DeviceGraph, quality: int, shots: int, is_spin_glass: bool, anneal_t: float,
                     anneal_h: float, repulsion_base: float, max_rounds: int = 1 << 20, jz_W=None):
    """sample_for_opencl (maxcut_tfim.py:148-186) on the device: draw rounds of
    candidates and score each round with the batched scoring kernel until a
    round does not beat the best so far. Returns (bool[n], value)."""
    n = dg.n
    _, _, cum = hamming_cdf(dg, quality, anneal_t, anneal_h, jz_W=jz_W)
    shots = ((max(1, shots >> 1) + 31) >> 5) << 5
    mpe = D.max_gpu_proc_elem(dg.device)
    G, L = D.geometry(shots, shots, mpe)
    best_solution = np.zeros(n, dtype=np.bool_)
    if is_spin_glass:
        _, en = dg.rescore(dg.pack(best_solution))
        best_energy = float(en.item())
    else:
        best_energy = 0.0
    seed = _current_seed()
    buf = None
    for round_ in range(max_rounds):
        buf = sample_batch(dg, cum, shots, repulsion_base, seed, round_, out=buf)
        _, be, bi = dg.calculate_cut(buf, shots, is_spin_glass, G, L, energies=False)
        energy = float(be.item())
        if energy > best_energy:
            b = int(bi.item())
            best_energy = float(np.float32(energy))
            best_solution = dg.unpack(buf[b * dg.n32 : (b + 1) * dg.n32])[0]
        else:
            break
    if is_spin_glass:
        cut, _ = dg.rescore(dg.pack(best_solution))
        best_energy = float(cut.item())
    return best_solution, float(best_energy)
