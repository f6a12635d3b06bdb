"""Drop-in ``solve_maxcut_bnb``: warm start from the heuristic, then exact
branch and bound (pyqrackising/solve_maxcut_bnb.py:208-321, loop :128-199).

Same signature (plus an optional ``batch_size``), defaults and 5-tuple
(bitstring, cut, (l, r), energy, certified). The traversal is the reference's:
a LIFO stack of partial assignments (int8, -1 free), popped ``batch_size`` at a
time (default os.cpu_count() ** 2, the reference's batch cap, so the same
nodes are visited in the same order); each batch is one ``pqi_bnb_eval``
launch (one GPU thread per node: bound, prune, leaf value or branch variable,
each summed in the reference's order); the host keeps the stack, the incumbent
and the pushes (warm value first, then its complement, so the complement is
popped first). A larger ``batch_size`` fills the GPU better and visits nodes in
another order; the certified value is the same.

Kept from the reference as it is: for spin glasses the bound is the cut bound
and the incumbent from the heuristic is the returned ``min_energy`` (the
negated energy, spin_glass_solver.py:727), exactly as the reference compares
them; the loop makes the same pruning decisions.
"""

from __future__ import annotations

import ctypes
import os
import time

import numpy as np
import torch

from . import _lib
from . import device as D
from .spin_glass_solver import spin_glass_solver
from .util import as_matrix, get_cut, int_to_bitstring


class _Evaluator:
    """Device buffers for batches of up to `cap` frontier nodes."""

    def __init__(self, dg: D.DeviceGraph, cap: int):
        self.dg = dg
        self.cap = cap
        dev = dg.device
        n = dg.n
        self.fv = torch.empty(n * cap, dtype=torch.int8, device=dev)
        self.ub = torch.empty(cap, dtype=torch.float64, device=dev)
        self.leaf = torch.empty(cap, dtype=torch.float64, device=dev)
        self.branch = torch.empty(cap, dtype=torch.int32, device=dev)
        self.state = torch.empty(cap, dtype=torch.int8, device=dev)
        self.h_fv = torch.empty(n * cap, dtype=torch.int8).pin_memory()
        self.h_leaf = torch.empty(cap, dtype=torch.float64).pin_memory()
        self.h_branch = torch.empty(cap, dtype=torch.int32).pin_memory()
        self.h_state = torch.empty(cap, dtype=torch.int8).pin_memory()

    def __call__(self, batch: np.ndarray, best_value: float, is_spin_glass: bool):
        """(state, leaf value, branch var) numpy arrays for the [count, n] batch."""
        count, n = batch.shape
        hv = self.h_fv[: n * count].numpy().reshape(n, count)
        hv[...] = batch.T
        self.fv[: n * count].copy_(self.h_fv[: n * count], non_blocking=True)
        _lib.call(
            "pqi_bnb_eval",
            D._ptr(self.dg.W),
            n,
            D._ptr(self.fv),
            count,
            ctypes.c_double(best_value),
            int(bool(is_spin_glass)),
            D._ptr(self.ub),
            D._ptr(self.leaf),
            D._ptr(self.branch),
            D._ptr(self.state),
            D.stream_ptr(),
        )
        self.h_state[:count].copy_(self.state[:count], non_blocking=True)
        self.h_leaf[:count].copy_(self.leaf[:count], non_blocking=True)
        self.h_branch[:count].copy_(self.branch[:count], non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return self.h_state[:count].numpy(), self.h_leaf[:count].numpy(), self.h_branch[:count].numpy()


def _branch_and_bound(dg, warm_theta, warm_energy, n, is_spin_glass, verbose=True, time_limit=None,
                      batch_size=None):
    """The reference's loop (solve_maxcut_bnb.py:128-199) with one device launch per batch.
    Returns (best bits, best value, certified)."""
    best_bits = np.asarray(warm_theta, dtype=np.bool_).copy()
    best_value = float(warm_energy)
    if verbose:
        print(f"Warm-start incumbent: {best_value:.6f}")
    cap = int(batch_size) if batch_size else (os.cpu_count() or 1) ** 2
    ev = _Evaluator(dg, cap)
    stack = np.empty((max(1024, 4 * cap), n), dtype=np.int8)
    stack[0] = -1
    top = 1
    t_start = time.monotonic()
    nodes_explored = 0
    nodes_pruned = 0
    while top:
        if time_limit is not None and (time.monotonic() - t_start) > time_limit:
            if verbose:
                print(f"Time limit reached. Nodes: {nodes_explored}, Pruned: {nodes_pruned}")
            return best_bits, best_value, False
        count = min(cap, top)
        batch = stack[top - count : top][::-1].copy()  # pop order: last pushed first
        top -= count
        nodes_explored += count
        state, leaf, branch = ev(batch, best_value, is_spin_glass)
        nodes_pruned += int(np.count_nonzero(state == 0))
        leaves = np.flatnonzero(state == 1)
        if leaves.size:
            vals = leaf[leaves]
            b = int(np.argmax(vals))
            if vals[b] > best_value:
                best_value = float(vals[b])
                best_bits = batch[leaves[b]] >= 1
                if verbose:
                    print(f"  New incumbent: {best_value:.6f}  (nodes: {nodes_explored})")
        interior = np.flatnonzero(state == 2)
        if interior.size:
            m = interior.size
            bv = branch[interior].astype(np.int64)
            warm = best_bits[bv].astype(np.int8)
            children = np.repeat(batch[interior], 2, axis=0)
            rows = np.arange(m)
            children[2 * rows, bv] = warm
            children[2 * rows + 1, bv] = 1 - warm
            if top + 2 * m > stack.shape[0]:
                grown = np.empty((max(2 * stack.shape[0], top + 2 * m), n), dtype=np.int8)
                grown[:top] = stack[:top]
                stack = grown
            stack[top : top + 2 * m] = children
            top += 2 * m
    if verbose:
        elapsed = time.monotonic() - t_start
        print(f"\nExact optimum: {best_value:.6f}")
        print(f"Nodes explored: {nodes_explored}  |  Pruned: {nodes_pruned}  |  Time: {elapsed:.3f}s")
    return best_bits, best_value, True


def solve_maxcut_bnb(
    G,
    best_guess=None,
    quality=None,
    shots=None,
    is_spin_glass=False,
    anneal_t=None,
    anneal_h=None,
    repulsion_base=None,
    is_maxcut_gpu=True,
    verbose=True,
    time_limit=None,
    gray_iterations=None,
    gray_seed_multiple=None,
    batch_size=None,
):
    nodes, G_m = as_matrix(G)
    G_m = np.asarray(G_m, dtype=np.float32)
    return _solve(nodes, G_m, spin_glass_solver, best_guess, quality, shots, is_spin_glass, anneal_t,
                  anneal_h, repulsion_base, is_maxcut_gpu, verbose, time_limit, gray_iterations,
                  gray_seed_multiple, batch_size)


def solve_maxcut_bnb_sparse(
    G,
    best_guess=None,
    quality=None,
    shots=None,
    is_spin_glass=False,
    anneal_t=None,
    anneal_h=None,
    repulsion_base=None,
    is_maxcut_gpu=True,
    verbose=True,
    time_limit=None,
    gray_iterations=None,
    gray_seed_multiple=None,
    batch_size=None,
):
    """The sparse-input B&B (pyqrackising/solve_maxcut_bnb_sparse.py:217-322):
    an nx.Graph or a scipy sparse matrix of upper-triangular stored entries (the
    reference's own layout, maxcut_tfim_util.py:533-542). Its bound, leaf and
    score loops over the stored entries (:33-121) are the dense loops over
    W = S + S^T, so the graph is expanded (on the device from 23 nodes) and the
    dense B&B runs; the warm start is spin_glass_solver_sparse. The branching
    score adds the same terms in another order (bit-equal for integer
    weights). A matrix that also stores lower-triangle entries is read as
    W = S + S^T throughout, as the sparse solver reads it."""
    from .sparse import _dense_operands, spin_glass_solver_sparse

    nodes, W, _ = _dense_operands(G)

    def heuristic(_W, **kwargs):
        return spin_glass_solver_sparse(G, **kwargs)

    return _solve(nodes, W, heuristic, best_guess, quality, shots, is_spin_glass, anneal_t, anneal_h,
                  repulsion_base, is_maxcut_gpu, verbose, time_limit, gray_iterations, gray_seed_multiple,
                  batch_size)


def _solve(nodes, W, heuristic, best_guess, quality, shots, is_spin_glass, anneal_t, anneal_h,
           repulsion_base, is_maxcut_gpu, verbose, time_limit, gray_iterations, gray_seed_multiple, batch_size):
    """solve_maxcut_bnb.py:253-321 on the dense matrix W (host array or device
    tensor); `heuristic` is the warm-start solver, called as the reference
    calls spin_glass_solver when best_guess is None."""
    n_qubits = len(nodes)

    if n_qubits < 3:
        if n_qubits == 0:
            return "", 0, ([], []), 0, True
        if n_qubits == 1:
            return "0", 0, (nodes, []), 0, True
        if n_qubits == 2:
            weight = W[0, 1]
            if weight < 0.0:
                return "00", 0, (nodes, []), weight, True
            return "01", weight, ([nodes[0]], [nodes[1]]), -weight, True

    cut_value = None
    energy_value = None
    if isinstance(best_guess, str):
        bitstring = best_guess
    elif isinstance(best_guess, int):
        bitstring = int_to_bitstring(best_guess, n_qubits)
    elif isinstance(best_guess, list):
        bitstring = "".join(["1" if b else "0" for b in best_guess])
    else:
        if verbose:
            print("Running PyQrackIsing heuristic...")
        kwargs = {}
        for key, val in (("quality", quality), ("shots", shots), ("anneal_t", anneal_t), ("anneal_h", anneal_h),
                         ("repulsion_base", repulsion_base), ("gray_iterations", gray_iterations),
                         ("gray_seed_multiple", gray_seed_multiple)):
            if val is not None:
                kwargs[key] = val
        kwargs["is_maxcut_gpu"] = is_maxcut_gpu
        t0 = time.monotonic()
        bitstring, cut_value, _, energy_value = heuristic(W, is_spin_glass=is_spin_glass, **kwargs)
        if verbose:
            print(f"Heuristic value: {cut_value:.6f}  ({time.monotonic()-t0:.3f}s)")

    dg = D.DeviceGraph(W)
    best_theta = np.array([b == "1" for b in list(bitstring)], dtype=np.bool_)
    if is_spin_glass:
        if energy_value is None:
            _, en = dg.rescore(dg.pack(best_theta))
            max_energy = float(en.item())
        else:
            max_energy = energy_value
    elif cut_value is None:
        cut, _ = dg.rescore(dg.pack(best_theta))
        max_energy = float(cut.item())
    else:
        max_energy = cut_value

    if verbose:
        print("Starting branch and bound...")

    best_theta, max_energy, certified = _branch_and_bound(
        dg, best_theta, max_energy, n_qubits, is_spin_glass, verbose=verbose, time_limit=time_limit,
        batch_size=batch_size,
    )

    bitstring, l, r = get_cut(best_theta, nodes)
    cut, en = dg.rescore(dg.pack(best_theta))
    if is_spin_glass:
        cut_value = float(cut.item())
        min_energy = -max_energy
    else:
        cut_value = max_energy
        min_energy = float(en.item())
    return bitstring, float(cut_value), (l, r), float(min_energy), certified
