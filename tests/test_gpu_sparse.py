"""Sparse-input entry points on the GPU against the reference's sparse path
(golden_sparse.npz) and against the dense entry points on the same graph."""

import importlib
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "golden_sparse.npz")


def test_sampler_init_reads_the_stored_rows():
    from scipy.sparse import csr_matrix

    import torch
    from pyqrackising_b200.device import DeviceGraph
    from pyqrackising_b200.sparse import sparse_to_dense

    MT = importlib.import_module("pyqrackising_b200.maxcut_tfim")
    z = np.load(GOLD)
    for i in range(int(z["count"])):
        _, W, S = sparse_to_dense(csr_matrix(z[f"U{i}"]))
        dg = DeviceGraph(W)
        J, deg, _ = MT.hamming_cdf(dg, 2, 8.0, 8.0, jz_W=torch.from_numpy(S).cuda())
        np.testing.assert_allclose(J.cpu().numpy(), z[f"J{i}"], rtol=1e-12, atol=1e-12)
        assert np.array_equal(deg.cpu().numpy(), z[f"deg{i}"])


def test_exhaustive_below_the_sparse_threshold():
    from scipy.sparse import csr_matrix

    from pyqrackising_b200 import maxcut_tfim_sparse

    z = np.load(GOLD)
    checked = 0
    for i in range(int(z["count"])):
        if f"exact{i}_0_val" not in z:
            continue
        G = csr_matrix(z[f"U{i}"])
        for spin in (0, 1):
            bits, val, _ = maxcut_tfim_sparse(G, is_spin_glass=bool(spin))
            ref_val = float(z[f"exact{i}_{spin}_val"])
            if ref_val < 0.0:
                assert bits == "0" * G.shape[0] and val == 0.0
            else:
                sol = "".join("1" if b else "0" for b in z[f"exact{i}_{spin}_sol"])
                assert bits == sol and val == pytest.approx(ref_val, rel=1e-6, abs=1e-6)
            checked += 1
    assert checked >= 2


def test_sparse_solver_equals_dense_solver_from_the_same_start(oracle_mod):
    from scipy.sparse import csr_matrix

    from pyqrackising_b200 import spin_glass_solver, spin_glass_solver_sparse

    O = oracle_mod
    z = np.load(GOLD)
    for i in (0, 1):
        U = z[f"U{i}"]
        W = U + U.T
        guess = [bool(b) for b in z[f"states{i}"][0]]
        for spin in (True, False):
            a = spin_glass_solver_sparse(csr_matrix(U), best_guess=guess, is_spin_glass=spin)
            b = spin_glass_solver(W, best_guess=guess, is_spin_glass=spin)
            assert a[0] == b[0] and a[1] == b[1] and a[3] == b[3]
            bits = np.array([c == "1" for c in a[0]])
            assert a[1] == pytest.approx(O.compute_cut(bits, W), rel=1e-9, abs=1e-6)


def test_sampling_path_returns_a_rescored_cut(oracle_mod):
    from scipy.sparse import csr_matrix

    from pyqrackising_b200 import maxcut_tfim_sparse

    O = oracle_mod
    MT = importlib.import_module("pyqrackising_b200.maxcut_tfim")
    z = np.load(GOLD)
    U = z["U1"]
    MT.set_seed(3)
    bits, val, (l, r) = maxcut_tfim_sparse(csr_matrix(U), quality=2)
    sol = np.array([c == "1" for c in bits])
    assert val == pytest.approx(O.compute_cut(sol, U + U.T), rel=1e-6, abs=1e-6)
    assert len(l) + len(r) == U.shape[0]
