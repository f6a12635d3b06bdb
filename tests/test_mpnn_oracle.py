"""The float64 oracle of the proposal network: its hand-written backward pass
agrees with central finite differences (no GPU)."""

import numpy as np

from oracle import mpnn_oracle as M


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    n = 30
    W = rng.standard_normal((n, n))
    W = np.triu(W, 1)
    W = W + W.T
    Ah, s = M.norm_adj(W)
    bits = rng.random(n) < 0.5
    F = M.features(bits, W, s)
    theta = M.init_params(3)
    t = np.zeros(n)
    t[[2, 5, 11]] = 1.0 / 3
    _, total = M.param_layout()
    idx = rng.choice(total, size=60, replace=False)
    num, ana = M.finite_difference_check(theta, F, Ah, t, idx)
    assert np.allclose(num, ana, rtol=1e-5, atol=1e-7), np.abs(num - ana).max()


def test_layout_matches_the_gpu_model():
    from pyqrackising_b200 import learned as L

    assert L.param_layout() == M.param_layout()
