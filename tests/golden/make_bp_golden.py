"""Golden marginals of the reference's belief propagation
(pyqrackising/spin_glass_solver.py:311-415), generated by importing the
reference in the build container (its checkout: $PQI_REFERENCE_ROOT, else
/root/reference):

    python tests/golden/make_bp_golden.py

Writes tests/golden/golden_bp.npz: a few small weighted graphs, the
bp_scale / damping used, and the reference's marginals."""

import os
import sys

import numpy as np

sys.path.insert(0, os.environ.get("PQI_REFERENCE_ROOT", "/root/reference"))
import importlib  # noqa: E402

ref = importlib.import_module("pyqrackising.spin_glass_solver")

HERE = os.path.dirname(os.path.abspath(__file__))
rng = np.random.default_rng(11)
out = {}
cases = [(12, 0.5, 1.0, 0.5), (20, 0.3, 0.5, 0.2), (30, 0.8, 2.0, 0.9)]
for i, (n, p, scale, damp) in enumerate(cases):
    W = np.triu((rng.random((n, n)) < p) * rng.standard_normal((n, n)), 1).astype(np.float32)
    W = W + W.T
    m = ref.belief_propagation_marginals_dense(W, n, scale, damp)
    out[f"W{i}"] = W
    out[f"params{i}"] = np.array([scale, damp])
    out[f"marg{i}"] = np.asarray(m, dtype=np.float64)
np.savez(os.path.join(HERE, "golden_bp.npz"), count=len(cases), **out)
print("wrote", len(cases), "cases")
