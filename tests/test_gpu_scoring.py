"""Tensor-core scoring (tcgen05) against exact values on ragged and full-size
shapes: n not a multiple of the 256-node tile or the 128-byte K block, batches
not a multiple of the 128-candidate tile, int8 and split-bf16 paths."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _exact_values(W, X, spin):
    x = np.where(X, 1.0, -1.0)
    Wd = W.astype(np.float64)
    q = np.einsum("bi,ij,bj->b", x, Wd, x)
    S = np.triu(Wd, 1).sum()
    return -q / 2 if spin else (2 * S - q) / 4


@pytest.mark.parametrize("n,shots", [(24, 1), (100, 37), (255, 128), (257, 129), (640, 300), (1000, 1000), (2048, 4096)])
@pytest.mark.parametrize("kind", ["int", "float"])
def test_tensor_core_scoring(n, shots, kind, oracle_mod):
    from pyqrackising_b200 import _lib
    from pyqrackising_b200 import workloads as wl
    from pyqrackising_b200.device import DeviceGraph

    O = oracle_mod
    rng = np.random.default_rng(n + shots)
    if kind == "int":
        W = wl.gnp_weighted(n, 0.5, seed=n, dist="uniform")
        W = np.where(W > 0, np.rint(W * 4) - 2, 0).astype(np.float32)  # integers in [-2, 2]
    else:
        W = wl.sherrington_kirkpatrick(n, seed=n)
    X = rng.random((shots, n)) < 0.5
    dg = DeviceGraph(W)
    assert dg.is_integer == (kind == "int")
    words = dg.pack(X)
    G, L = O.cut_geometry(shots, 148)
    for spin in (0, 1):
        e, be, bi = dg.calculate_cut(words, shots, spin, G, L)
        got = e.cpu().numpy().astype(np.float64)
        exact = _exact_values(W, X, spin)
        if kind == "int":
            assert np.array_equal(got, exact), np.abs(got - exact).max()
            ref = O.select(exact.astype(np.float32), G, L)
            assert (float(be.item()), int(bi.item())) == (float(ref[0]), ref[1])
        else:
            tol = 1e-5 * np.abs(W.astype(np.float64)).sum() / 2
            assert np.all(np.abs(got - exact) <= tol), np.abs(got - exact).max() / tol
        # same answer from the CUDA-core path (1), single CTAs (2), CTA pairs
        # (3, the default's form), the split-bf16 form of float weights (4) and
        # single CTAs that expand the candidates themselves (5); the default
        # (0) scores float weights as fixed-point digit planes
        for path in (1, 2, 3, 4, 5):
            _lib.call("pqi_score_set_path", path)
            try:
                e1, be1, bi1 = dg.calculate_cut(words, shots, spin, G, L)
            finally:
                _lib.call("pqi_score_set_path", 0)
            if kind == "int":
                assert torch.equal(e1, e) and int(bi1.item()) == int(bi.item()), path
            else:
                assert np.all(np.abs(e1.cpu().numpy().astype(np.float64) - exact) <= tol), path
