"""Host-side logic of the drop-in (no GPU): launch geometry, pair decoding,
best_guess parsing, result formatting."""

import importlib

import numpy as np

from pyqrackising_b200 import device as D
from pyqrackising_b200 import util

S = importlib.import_module("pyqrackising_b200.spin_glass_solver")


def test_geometry_matches_setup_opencl(oracle_mod):
    for n in (3, 24, 31, 64, 100, 2048, 8192):
        for mpe in (1, 7, 148, 4096):
            assert D.geometry(min(32, n), n, mpe) == oracle_mod.flip_geometry(n, mpe)
    assert D.geometry(1, 148, 148) == (148, 1)
    assert D.geometry(2048, 2048, 148) == (160, 32)


def test_pair_decode_matches_reference_loop(oracle_mod):
    for n in (2, 3, 10, 57):
        c = 0
        for k in range(n):
            for l in range(k + 1, n):
                assert S.pair_decode(c, n) == (k, l) == oracle_mod.pair_decode(c, n)
                c += 1


def test_pair_decode_64_bit_indices():
    """The closed form at sizes whose pair count exceeds int32 (the
    compressed-row double pass reports 64-bit pair indices)."""
    rng = np.random.default_rng(0)
    for n in (46341, 46342, 200000, 1 << 20):
        total = n * (n - 1) // 2
        for c in [0, 1, total - 1, total // 2] + [int(x) for x in rng.integers(0, total, 50)]:
            k, l = S.pair_decode(c, n)
            assert 0 <= k < l < n and k * (n - 1) - k * (k - 1) // 2 + (l - k - 1) == c


def test_best_guess_parsing():
    n = 8
    assert util.parse_best_guess("10110000", n).tolist() == [True, False, True, True, False, False, False, False]
    assert util.parse_best_guess(13, n).tolist() == [True, False, True, True, False, False, False, False]
    assert util.parse_best_guess([1, 0, 1], 3).tolist() == [True, False, True]
    assert util.parse_best_guess(None, n) is None
    assert util.parse_best_guess(np.int64(3), n) is None  # the reference only accepts a Python int


def test_get_cut():
    bs, l, r = util.get_cut(np.array([1, 0, 1], bool), ["a", "b", "c"])
    assert bs == "101" and l == ["b"] and r == ["a", "c"]


def test_bp_marginals_match_reference_golden():
    """The reference's loopy BP stays at its zero starting messages: marginals
    and the warm-start partition match the reference's own outputs."""
    import importlib
    import os

    SG = importlib.import_module("pyqrackising_b200.spin_glass_solver")
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_bp.npz"))
    for i in range(int(z["count"])):
        W = z[f"W{i}"]
        scale, damp = z[f"params{i}"]
        m = SG.belief_propagation_marginals_dense(W, W.shape[0], scale, damp)
        assert np.array_equal(m, z[f"marg{i}"])
        assert not SG.bp_warm_start_dense(W, W.shape[0], scale, damp).any()
