"""Golden results of the reference's exact branch-and-bound solver, generated by
importing the reference in the build container (PYTHONPATH=/root/reference):

    python tests/golden/make_bnb_golden.py

Writes tests/golden/golden_bnb.npz: per case the dense float32 matrix W, the
warm start (best_guess bit string), the objective (cut or spin glass), the
reference's returned bit string, cut, energy and certified flag
(solve_maxcut_bnb.py:208-321, run with verbose=False), the same for the sparse
solver on the upper-triangular CSR of W (solve_maxcut_bnb_sparse.py:217-322,
keys *_sparse_*), and the batch cap the reference used here (os.cpu_count() ** 2,
which fixes its traversal order)."""

import importlib
import os
import sys

import numpy as np
from scipy.sparse import csr_matrix

sys.path.insert(0, "/root/reference")
bnb = importlib.import_module("pyqrackising.solve_maxcut_bnb")
bnbs = importlib.import_module("pyqrackising.solve_maxcut_bnb_sparse")

HERE = os.path.dirname(os.path.abspath(__file__))
rng = np.random.default_rng(41)


def sym(U):
    U = np.triu(U, 1).astype(np.float32)
    return (U + U.T).astype(np.float32)


def regular3(n):
    # random 3-regular multigraph-free pairing, +-1 weights
    while True:
        stubs = rng.permutation(np.repeat(np.arange(n), 3))
        a, b = stubs[0::2], stubs[1::2]
        if np.any(a == b):
            continue
        key = np.minimum(a, b) * n + np.maximum(a, b)
        if np.unique(key).size != key.size:
            continue
        U = np.zeros((n, n), dtype=np.float32)
        U[np.minimum(a, b), np.maximum(a, b)] = rng.choice([-1.0, 1.0], size=a.size)
        return sym(U)


cases = [
    ("reg16_cut", regular3(16), False),
    ("reg16_spin", regular3(16), True),
    ("gnp14_uniform_cut", sym(np.where(rng.random((14, 14)) < 0.5, 1.0 - rng.random((14, 14)), 0.0)), False),
    ("gnp14_normal_spin", sym(np.where(rng.random((14, 14)) < 0.5, rng.standard_normal((14, 14)), 0.0)), True),
    ("int12_cut", sym(rng.choice([-2.0, -1.0, 0.0, 1.0, 3.0], size=(12, 12))), False),
    ("int12_spin", sym(rng.choice([-2.0, -1.0, 0.0, 1.0, 3.0], size=(12, 12))), True),
    ("ones10_cut", sym(np.ones((10, 10))), False),
]
out = {"names": np.array([c[0] for c in cases]), "batch_cap": np.int64((os.cpu_count() or 1) ** 2)}
for name, W, spin in cases:
    n = W.shape[0]
    guess = "".join("1" if b else "0" for b in (rng.random(n) < 0.5))
    bits, cut, _, energy, certified = bnb.solve_maxcut_bnb(W, best_guess=guess, is_spin_glass=spin, verbose=False)
    out[f"{name}_W"] = W
    out[f"{name}_guess"] = np.array(guess)
    out[f"{name}_spin"] = np.int64(spin)
    out[f"{name}_bits"] = np.array(bits)
    out[f"{name}_cut"] = np.float64(cut)
    out[f"{name}_energy"] = np.float64(energy)
    out[f"{name}_certified"] = np.int64(bool(certified))
    print(name, bits, cut, energy, certified)
    sb, sc, _, se, scert = bnbs.solve_maxcut_bnb_sparse(csr_matrix(np.triu(W, 1)), best_guess=guess,
                                                         is_spin_glass=spin, verbose=False)
    out[f"{name}_sparse_bits"] = np.array(sb)
    out[f"{name}_sparse_cut"] = np.float64(sc)
    out[f"{name}_sparse_energy"] = np.float64(se)
    out[f"{name}_sparse_certified"] = np.int64(bool(scert))
    print(name, "sparse", sb, sc, se, scert)
np.savez_compressed(os.path.join(HERE, "golden_bnb.npz"), **out)
