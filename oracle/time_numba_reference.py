"""TEST INFRASTRUCTURE ONLY: time the reference's own numba CPU scoring next to
the oracle's restatement of it (oracle/numba_port.py), on the same cores.

Build container only (the reference checkout is not present elsewhere):

    PQI_REFERENCE_ROOT=/path/to/reference NUMBA_CACHE_DIR=/tmp/numba_cache \
        python oracle/time_numba_reference.py [candidates]

Workload: the bench's graph (ER G(2048, 0.5), unit weights, float32) and a
sample of uniform random candidates. The reference side is its
``compute_cut_diff_between`` (``pyqrackising/maxcut_tfim_util.py:445-461``),
imported unmodified, called once per candidate inside a numba ``prange`` as
``sample_measurement`` does (``pyqrackising/maxcut_tfim.py:77-136``). Prints
one JSON line: candidates/s of each side (median of 5 runs after a warm-up),
numba's thread count and whether the values agree.
"""

from __future__ import annotations

import importlib
import json
import os
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)
sys.path.insert(0, os.environ.get("PQI_REFERENCE_ROOT", "/root/reference"))
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache")


def main():
    from numba import get_num_threads, njit, prange

    from oracle import numba_port as P
    from pyqrackising_b200 import workloads as wl

    mu = importlib.import_module("pyqrackising.maxcut_tfim_util")
    ref_cd = mu.compute_cut_diff_between

    @njit(parallel=True)
    def ref_batch(base, cands, G, out):
        n = G.shape[0]
        for b in prange(cands.shape[0]):
            out[b] = ref_cd(base, cands[b], G, n)

    B = int(sys.argv[1]) if len(sys.argv) > 1 else 1024
    W = wl.erdos_renyi(2048, 0.5, seed=1)
    X = np.random.default_rng(1000).random((B, 2048)) < 0.5
    base = np.zeros(2048, dtype=np.bool_)
    out = np.empty(B, dtype=np.float64)
    ref_batch(base, X[:2], W, out[:2])
    P.warm()
    res = {}
    for name, fn in (("reference", lambda: ref_batch(base, X, W, out)), ("port", lambda: P.score_batch(X, W))):
        ts = []
        for _ in range(5):
            t0 = time.perf_counter()
            fn()
            ts.append(time.perf_counter() - t0)
        res[name] = B / float(np.median(ts))
    ref_vals = out.copy()
    agree = bool(np.array_equal(ref_vals, P.score_batch(X, W)))
    print(json.dumps({"workload": f"ER G(2048, 0.5) unit weights, {B} random candidates",
                      "reference_candidates_per_s": res["reference"], "port_candidates_per_s": res["port"],
                      "numba_threads": get_num_threads(), "values_agree": agree}))


if __name__ == "__main__":
    main()
