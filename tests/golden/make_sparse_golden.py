"""Golden vectors of the reference's sparse path, generated by importing the
reference in the build container (its checkout: $PQI_REFERENCE_ROOT, else
/root/reference):

    python tests/golden/make_sparse_golden.py

Writes tests/golden/golden_sparse.npz: upper-triangular CSR graphs (as dense
upper matrices), the reference's sparse J_eff / degrees
(maxcut_tfim_sparse.py:204-224), sparse cut and energy of random states
(maxcut_tfim_util.py:350-371), and the exhaustive sparse solutions below the
sparse threshold (maxcut_tfim_sparse.py:310-371)."""

import importlib
import os
import sys

import numpy as np
from scipy.sparse import csr_matrix

sys.path.insert(0, os.environ.get("PQI_REFERENCE_ROOT", "/root/reference"))
ms = importlib.import_module("pyqrackising.maxcut_tfim_sparse")
mu = importlib.import_module("pyqrackising.maxcut_tfim_util")

HERE = os.path.dirname(os.path.abspath(__file__))
rng = np.random.default_rng(23)
out = {}
cases = [(40, 0.2, "normal"), (60, 0.1, "pm1"), (22, 0.4, "uniform"), (18, 0.5, "pm1")]
for i, (n, p, dist) in enumerate(cases):
    mask = np.triu(rng.random((n, n)) < p, 1)
    if dist == "normal":
        vals = rng.standard_normal((n, n))
    elif dist == "pm1":
        vals = rng.choice([-1.0, 1.0], size=(n, n))
    else:
        vals = 1.0 - rng.random((n, n))
    U = np.where(mask, vals, 0.0).astype(np.float32)
    G = csr_matrix(U)
    J, deg = ms.init_J_and_z(G, 5.0)
    states = rng.random((6, n)) < 0.5
    cuts = [mu.compute_cut_sparse(s, G.data, G.indptr, G.indices, n) for s in states]
    ens = [mu.compute_energy_sparse(s, G.data, G.indptr, G.indices, n) for s in states]
    out[f"U{i}"] = U
    out[f"J{i}"] = np.asarray(J, dtype=np.float64)
    out[f"deg{i}"] = np.asarray(deg, dtype=np.int64)
    out[f"states{i}"] = states
    out[f"cut{i}"] = np.asarray(cuts, dtype=np.float64)
    out[f"energy{i}"] = np.asarray(ens, dtype=np.float64)
    if n < mu.heuristic_threshold_sparse:
        for spin in (0, 1):
            sol, val = (ms.exact_spin_glass if spin else ms.exact_maxcut)(G.data, G.indptr, G.indices)
            out[f"exact{i}_{spin}_sol"] = np.asarray(sol, dtype=np.bool_)
            out[f"exact{i}_{spin}_val"] = np.float64(val)
np.savez(os.path.join(HERE, "golden_sparse.npz"), count=len(cases), **out)
print("wrote", len(cases), "cases")
