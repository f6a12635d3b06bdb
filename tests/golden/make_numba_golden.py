"""Golden values of the reference's CPU candidate scoring, made by importing
the reference itself (build container only):

    NUMBA_CACHE_DIR=/tmp/numba_cache python tests/golden/make_numba_golden.py

For each instance: random base and candidate states, and the reference's
``compute_cut_diff_between(base, cand, G_m, n)``
(``pyqrackising/maxcut_tfim_util.py:445-461``) for every pair, plus the values
against the all-false base (the cuts ``sample_measurement`` starts from,
``pyqrackising/maxcut_tfim.py:77-136``). ``tests/test_numba_port.py`` checks
the oracle's restatement (``oracle/numba_port.py``) against them bit for bit.
Writes ``tests/golden/golden_numba_cutdiff.npz``.
"""

from __future__ import annotations

import importlib
import os
import sys

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REFERENCE = os.environ.get("PQI_REFERENCE_ROOT", "/root/reference")
sys.path.insert(0, REPO)
sys.path.insert(0, REFERENCE)
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache")

from pyqrackising_b200 import workloads as wl  # noqa: E402


def main():
    mu = importlib.import_module("pyqrackising.maxcut_tfim_util")
    out = {}
    cases = (
        ("er300", wl.erdos_renyi(300, 0.5, seed=11)),
        ("sk200", wl.sherrington_kirkpatrick(200, seed=12)),
        ("gnp257", wl.gnp_weighted(257, 0.1, seed=13, dist="normal")),
    )
    for name, W in cases:
        n = W.shape[0]
        rng = np.random.default_rng(n)
        base = rng.random((8, n)) < 0.5
        cand = rng.random((8, n)) < 0.5
        vals = np.array([mu.compute_cut_diff_between(base[i], cand[i], W, n) for i in range(8)])
        zero = np.zeros(n, dtype=np.bool_)
        cuts = np.array([mu.compute_cut_diff_between(zero, cand[i], W, n) for i in range(8)])
        out[f"{name}_W"] = W
        out[f"{name}_base"] = base
        out[f"{name}_cand"] = cand
        out[f"{name}_values"] = vals
        out[f"{name}_cuts"] = cuts
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_numba_cutdiff.npz"), **out)


if __name__ == "__main__":
    main()
