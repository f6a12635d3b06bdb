"""Drop-in ``spin_glass_solver`` on the B200 path.

Same signature, defaults and return tuple as the reference
(``pyqrackising/spin_glass_solver.py:424-727``). The local search follows the
reference's GPU branch move for move:

1. single-bit-flip passes until none improves (``:608-627``),
2. then one double-bit-flip pass (``:629-648``), back to 1 if it improved,
3. then one parallel Gray-code search (``:650-668``), back to 1 if it improved,
4. else stop (the post-reheat phase, ``:670-717``, re-runs passes 1 and 2 on
   the unchanged state on this branch, so it cannot improve and is skipped).

Every selection uses the reference's launch geometry, so ties pick the same
node (``include/pqi.h``). Differences, all deliberate:

* The gains stay on the device and are updated in O(n) per accepted flip; the
  whole run of single flips is one kernel launch (``pqi_single_descent``)
  instead of one host round trip per flip.
* ``gray_seed_multiple`` sets the number of parallel Gray seeds on the GPU (the
  reference's GPU branch ignores it and uses MAX_GPU_PROC_ELEM, which is the
  default here too).
* Returned cut and energy are float64 re-scorings of the returned bit string.
  The reference returns its running total for one of them (``:720-725``),
  which drifts after an accepted Gray move (the gray kernel reports half the
  change, ``kernels.cl:974-976``).
* ``is_maxcut_gpu`` is accepted and ignored: there is no CPU path.
* ``bp_scale`` runs the reference's belief-propagation warm start, whose
  messages stay at their zero starting point (see
  ``belief_propagation_marginals_dense``): its all-False partition competes with
  the TFIM sample exactly as in the reference.
"""

from __future__ import annotations

import math

import numpy as np
import torch

from . import device as D
from .maxcut_tfim import _maxcut_tfim, maxcut_tfim  # noqa: F401
from .util import HEURISTIC_THRESHOLD, as_matrix, get_cut, parse_best_guess


def pair_decode(c: int, n: int):
    """Linear pair index -> (k, l), the reference's enumeration
    (spin_glass_solver.py:224-234): pair (k, l), k < l, has index
    k(n-1) - k(k-1)/2 + (l-k-1). Closed form, exact for 64-bit indices."""
    c = int(c)
    base = lambda k: k * (n - 1) - (k * (k - 1)) // 2  # noqa: E731
    # largest k with base(k) <= c, from the quadratic, then corrected exactly
    b = 2 * n - 1
    k = max(0, min(n - 2, int((b - math.isqrt(max(0, b * b - 8 * c))) // 2)))
    while k > 0 and base(k) > c:
        k -= 1
    while k + 1 <= n - 2 and base(k + 1) <= c:
        k += 1
    return k, c - base(k) + k + 1


class SearchStats:
    """Counters of one solver run (moves accepted per kind, device flips)."""

    def __init__(self):
        self.single = 0
        self.double = 0
        self.gray = 0
        self.rounds = 0
        self.trace = []

    def as_dict(self):
        return {"single": self.single, "double": self.double, "gray": self.gray, "rounds": self.rounds}


GRAY_NODE_LIMIT = 131072  # maxcut_tfim_util.py:11: no GPU Gray search above it


def local_search(dg, theta, is_spin_glass: bool, gray_iterations: int, gray_seeds: int,
                 mpe: int, max_energy: float, stats: SearchStats | None = None, record_trace: bool = False,
                 max_rounds: int | None = None):
    """Run the reference's GPU-branch loop from bool[n] `theta` on a prepared
    graph: a dense ``device.DeviceGraph`` or a CSR ``sparse.SparseDeviceGraph``
    (the same methods). Above GRAY_NODE_LIMIT nodes the Gray stage is skipped,
    as the reference's GPU branch has no Gray kernel there
    (spin_glass_solver_sparse.py:628,752). Returns (device words of the final
    state, running max_energy)."""
    n = dg.n
    words = dg.pack(theta)
    _, g64 = dg.gains(words)
    Gf, Lf = D.geometry(min(D.WORK_GROUP_MULTIPLE, n), n, mpe)
    iters_bound = (gray_iterations + gray_seeds - 1) // gray_seeds
    budget = max(4 * n, 1024)
    trace = torch.empty(budget, dtype=torch.int32, device=dg.device) if record_trace else None
    spin = bool(is_spin_glass)
    rounds = 0
    while True:
        rounds += 1
        if max_rounds is not None and rounds > max_rounds:
            break
        # 1. single flips, all on the device
        while True:
            esum, flips, rc = dg.single_descent(words, g64, spin, Gf, Lf, budget, trace)
            nf = int(flips.item())
            max_energy += float(esum.item())
            if stats is not None:
                stats.single += nf
                if record_trace and nf:
                    stats.trace.extend(("single", int(k)) for k in trace[:nf].tolist())
            if rc != 3:  # PQI_ETIMEOUT: budget used up, keep going
                break
        # 2. double flips
        if n >= 2:
            be, bi = dg.double_bit_flips(words, g64, spin, Gf, Lf, improving=True)
            e = float(be.item())
            if e > 0.0:
                k, l = pair_decode(int(bi.item()), n)
                dg.apply_flip(words, g64, k, l)
                max_energy += e
                if stats is not None:
                    stats.double += 1
                    if record_trace:
                        stats.trace.append(("double", k, l))
                continue
        # 3. parallel Gray-code search
        if n > GRAY_NODE_LIMIT:
            break
        tout, eout = dg.gray(words, g64, spin, iters_bound, gray_seeds)
        be, bi = dg.select(eout, gray_seeds, 1)
        e = float(be.item())
        if e > 0.0:
            bx = int(bi.item())
            row = tout[bx * 2 * dg.n64 : bx * 2 * dg.n64 + dg.n32].clone()
            if n & 31:
                row[-1] &= (1 << (n & 31)) - 1  # bits >= n are padding (the reference unpacks bits < n)
            words[: dg.n32] = row
            _, g64 = dg.gains(words)
            max_energy += e
            if stats is not None:
                stats.gray += 1
                if record_trace:
                    stats.trace.append(("gray", bx))
            continue
        break
    if stats is not None:
        stats.rounds = rounds
    return words, max_energy


def belief_propagation_marginals_dense(G_m, n, bp_scale=1.0, damping=0.5):
    """Per-node marginals of the reference's loopy belief propagation
    (spin_glass_solver.py:311-415).

    The reference starts every message at 0 and updates
    m <- damping * m + (1 - damping) * artanh(clip(tanh(w) * tanh(h))), where h is
    a sum of the node's other incoming messages. With every message 0, h = 0,
    tanh(h) = 0, the product and its artanh are 0, and the damped message stays
    0; so every message is exactly 0 after any number of iterations, for every
    weight set and damping, and the marginals tanh(sum of messages) are exactly
    0. This returns that result without iterating."""
    return np.zeros(int(n), dtype=np.float64)


def bp_warm_start_dense(G_m, n, bp_scale=1.0, damping=0.5):
    """Partition from the BP marginals: marginal > 0 (spin_glass_solver.py:418-421)."""
    return belief_propagation_marginals_dense(G_m, n, bp_scale, damping) > 0.0


def spin_glass_solver(
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
    nodes, G_m = as_matrix(G)
    return _spin_glass_solver(nodes, G_m, quality, shots, best_guess, is_maxcut_gpu, is_spin_glass, anneal_t,
                              anneal_h, repulsion_base, gray_iterations, gray_seed_multiple, bp_scale, bp_damping)


def _spin_glass_solver(nodes, G_m, quality, shots, best_guess, is_maxcut_gpu, is_spin_glass, anneal_t, anneal_h,
                       repulsion_base, gray_iterations, gray_seed_multiple, bp_scale, bp_damping,
                       threshold=HEURISTIC_THRESHOLD, jz_matrix=None, graph=None):
    """spin_glass_solver on a dense symmetric matrix; `threshold` and
    `jz_matrix` as in maxcut_tfim._maxcut_tfim (the sparse entry point's
    values differ). `graph`: an already prepared graph to search on instead
    of G_m (the sparse entry points' compressed rows, with G_m None; only for
    graphs above `threshold` and 2 nodes)."""
    n_qubits = len(nodes)

    if n_qubits < 3:
        if n_qubits == 0:
            return "", 0, ([], []), 0
        if n_qubits == 1:
            return "0", 0, (nodes, []), 0
        if n_qubits == 2:
            weight = G_m[0, 1]
            if weight < 0.0:
                return "00", 0, (nodes, []), weight
            return "01", weight, ([nodes[0]], [nodes[1]]), -weight

    if n_qubits < threshold:
        best_guess = None

    theta = parse_best_guess(best_guess, n_qubits)
    cut_value = None
    # prepared once, shared by the seed sampler and the search
    dg = graph if graph is not None else D.DeviceGraph(G_m)
    if theta is None:
        bitstring, cut_value, _ = _maxcut_tfim(
            list(range(n_qubits)), G_m, quality, shots, is_spin_glass, anneal_t, anneal_h, repulsion_base,
            threshold=threshold, jz_matrix=jz_matrix, dg=dg,
        )
        if bp_scale is not None and n_qubits >= threshold:
            # keep whichever of the BP partition and the sample scores higher
            # (spin_glass_solver.py:493-523)
            bp_theta = bp_warm_start_dense(G_m, n_qubits, bp_scale, bp_damping)
            sample_theta = np.array([b == "1" for b in bitstring], dtype=np.bool_)
            cb, eb = dg.rescore(dg.pack(bp_theta))
            cs, es = dg.rescore(dg.pack(sample_theta))
            bp_energy = float(eb.item()) if is_spin_glass else float(cb.item())
            sample_energy = float(es.item()) if is_spin_glass else float(cs.item())
            if bp_energy > sample_energy:
                bitstring = "".join("1" if b else "0" for b in bp_theta)
                cut_value = bp_energy if not is_spin_glass else None
        theta = np.array([b == "1" for b in bitstring], dtype=np.bool_)

    words = dg.pack(theta)
    cut0, en0 = dg.rescore(words)
    if is_spin_glass:
        max_energy = float(en0.item())
    elif cut_value is None:
        max_energy = float(cut0.item())
    else:
        max_energy = cut_value

    if n_qubits < threshold:
        bitstring, l, r = get_cut(theta, nodes)
        if is_spin_glass:
            cut_value = float(cut0.item())
            min_energy = -max_energy
        else:
            cut_value = max_energy
            min_energy = float(en0.item())
        return bitstring, float(cut_value), (l, r), float(min_energy)

    if gray_iterations is None:
        gray_iterations = n_qubits * n_qubits
    mpe = D.max_gpu_proc_elem(dg.device)
    seeds = int(gray_seed_multiple) if gray_seed_multiple is not None else mpe

    words, max_energy = local_search(dg, theta, is_spin_glass, int(gray_iterations), seeds, mpe, max_energy)

    best = dg.unpack(words)[0]
    cut, en = dg.rescore(words)
    bitstring, l, r = get_cut(best, nodes)
    cut_value = float(cut.item())
    min_energy = -float(en.item()) if is_spin_glass else float(en.item())
    return bitstring, cut_value, (l, r), min_energy
