"""TEST INFRASTRUCTURE ONLY: the reference's CPU (numba) candidate scoring,
restated for the CPU baseline.

Only ``tests/`` and ``bench.py``'s CPU-baseline and reference legs may import
this module; the product never does.

The reference scores candidate bit strings on its CPU path in
``sample_measurement`` (``pyqrackising/maxcut_tfim.py:77-136``): one numba
``prange`` over worker slots, each scoring its shots one after another with
``compute_cut_diff_between(solutions[i], sample, G_m, n)``
(``pyqrackising/maxcut_tfim_util.py:445-461``): a float64 sum over the upper
triangle u < v of +W_uv where the pair becomes cut, -W_uv where it stops being
cut, nothing elsewhere. ``score_batch`` below applies that per-candidate sum
to a batch under ``prange`` (numba's thread pool, ``NUMBA_NUM_THREADS``
threads, default all cores) and returns the values; ``select_first_max``
takes the first maximum as ``np.argmax`` does (``maxcut_tfim.py:115``).

With the all-false state as the base (``sample_measurement`` starts every slot
from it, ``maxcut_tfim.py:83``) a candidate's value is its cut. The sums run
in the reference's order with the reference's types (float32 weights, float64
accumulator), so values equal the reference function's bit for bit
(``tests/test_numba_port.py`` against ``tests/golden/golden_numba_cutdiff.npz``,
made by ``tests/golden/make_numba_golden.py`` from the reference itself).
"""

from __future__ import annotations

import os

import numpy as np

_fns = None


def available() -> bool:
    try:
        import numba  # noqa: F401
    except ImportError:
        return False
    return True


def threads() -> int:
    import numba

    return int(numba.get_num_threads())


def _compile():
    global _fns
    if _fns is not None:
        return _fns
    os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(os.path.dirname(os.path.abspath(__file__)), "_numba_cache"))
    from numba import njit, prange

    @njit(cache=True)
    def cut_change(base, cand, G, n):
        # maxcut_tfim_util.py:445-461: u-major, then v > u; a pair counts when
        # its cut status differs between the two strings
        total = 0.0
        for u in range(n):
            row = G[u]
            bu = base[u]
            cu = cand[u]
            for v in range(u + 1, n):
                was_cut = bu != base[v]
                now_cut = cu != cand[v]
                if was_cut != now_cut:
                    w = row[v]
                    if now_cut:
                        total += w
                    else:
                        total -= w
        return total

    @njit(parallel=True, cache=True)
    def score_batch_impl(base, cands, G, out):
        n = G.shape[0]
        for b in prange(cands.shape[0]):
            out[b] = cut_change(base, cands[b], G, n)

    _fns = (cut_change, score_batch_impl)
    return _fns


def cut_change(base, cand, G) -> float:
    """compute_cut_diff_between(base, cand, G, n) restated."""
    f, _ = _compile()
    G = np.ascontiguousarray(G, dtype=np.float32)
    return float(f(np.asarray(base, np.bool_), np.asarray(cand, np.bool_), G, G.shape[0]))


def score_batch(cands, G, base=None) -> np.ndarray:
    """Values of every candidate row of ``cands`` (bool[B, n]) against ``base``
    (default all-false: the cut), in parallel over candidates."""
    _, f = _compile()
    G = np.ascontiguousarray(G, dtype=np.float32)
    cands = np.ascontiguousarray(cands, dtype=np.bool_)
    if base is None:
        base = np.zeros(G.shape[0], dtype=np.bool_)
    out = np.empty(cands.shape[0], dtype=np.float64)
    f(np.asarray(base, np.bool_), cands, G, out)
    return out


def select_first_max(values) -> tuple[float, int]:
    i = int(np.argmax(values))
    return float(values[i]), i


def warm():
    """Compile (or load from the cache) before anything is timed."""
    G = np.zeros((4, 4), dtype=np.float32)
    score_batch(np.zeros((2, 4), dtype=np.bool_), G)
