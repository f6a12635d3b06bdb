"""The CPU oracle against the reference's own outputs (golden fixtures).

* ``kcl_*`` fixtures were produced by the reference's kernels.cl run on the host
  (oracle/_ref); the C restatement must reproduce them bit for bit.
* ``ref_*`` fixtures were produced by the reference's numba code; the oracle's
  float64 objectives must agree to float64 rounding.
"""

import numpy as np
import pytest

from conftest import golden_names, load_golden

NAMES = golden_names()


@pytest.mark.parametrize("name", NAMES)
def test_objectives_match_reference_numba(name, oracle_mod):
    O = oracle_mod
    d = load_golden(name)
    W, th = d["W"], d["theta"]
    # the reference's compute_cut multiplies a bool matrix by float32 W and sums in
    # float32 (maxcut_tfim_util.py:329-331): float32 rounding, exact on integers
    assert abs(O.compute_cut(th, W) - float(d["ref_compute_cut"])) <= 2e-6 * np.abs(W).sum() + 1e-12
    assert abs(O.compute_energy(th, W) - float(d["ref_compute_energy"])) <= 2e-6 * np.abs(W).sum() + 1e-12
    # packing (convert_bool_to_uint)
    assert np.array_equal(O.pack32(th), d["ref_convert_bool_to_uint"])
    # flip gains: oracle's single-flip values (x1) vs the reference CPU twin's compute_cut_diff
    vals = O.single_values(W, O.pack32(th), 0).astype(np.float64)
    tol = 1e-5 * np.abs(W).sum(axis=1) + 1e-6
    assert np.all(np.abs(vals - d["ref_cut_diff"]) <= tol)
    # pair gains: the kernel's double-flip value vs compute_cut_diff_2
    for (k, l), ref in zip(d["pairs"], d["ref_cut_diff_2"]):
        got = O.double_value(W, O.pack32(th), int(k), int(l))
        assert abs(got - ref) <= 1e-5 * (np.abs(W[k]).sum() + np.abs(W[l]).sum()) + 1e-6
    # gray_mutation seeds and the cut change against them
    for s, ref in zip(d["ref_gray_mutation"], d["ref_cut_diff_between"]):
        assert O.compute_cut_diff_between(th, s, W) == pytest.approx(float(ref), rel=1e-9, abs=1e-9)


@pytest.mark.parametrize("name", NAMES)
def test_kernel_restatement_matches_reference_kernels(name, oracle_mod):
    O = oracle_mod
    d = load_golden(name)
    W, th, spin = d["W"], d["theta"], int(d["is_spin_glass"])
    n = W.shape[0]
    th32 = O.pack32(th)
    for mpe in (148, 4096):
        G, L = O.flip_geometry(n, mpe)
        e, i = O.single_select(W, th32, spin, G, L)
        assert (np.float32(e), i) == (np.float32(d[f"kcl_single_{mpe}"][0]), int(d[f"kcl_single_{mpe}"][1]))
        _, _, ge, gi = O.select(O.single_values(W, th32, spin), G, L, with_groups=True)
        assert np.array_equal(ge.astype(np.float64), d[f"kcl_single_{mpe}_groups"][0])
        assert np.array_equal(gi.astype(np.float64), d[f"kcl_single_{mpe}_groups"][1])
        e, c = O.double_select(W, th32, spin, G, L)
        assert (np.float32(e), c) == (np.float32(d[f"kcl_double_{mpe}"][0]), int(d[f"kcl_double_{mpe}"][1]))
    X = d["cut_candidates"]
    G, L = O.cut_geometry(X.shape[0], 148)
    e, i = O.cut_select(W, O.pack32(X), X.shape[0], spin, G, L)
    assert (np.float32(e), i) == (np.float32(d["kcl_cut_148"][0]), int(d["kcl_cut_148"][1]))
    for S in (148, 512):
        T = int(d[f"kcl_gray_{S}_T"])
        tout, eout, oob = O.gray(W, O.pack64(th), spin, T, S)
        assert oob == 0
        assert np.array_equal(tout, d[f"kcl_gray_{S}_theta"])
        assert np.array_equal(eout.view(np.uint32), d[f"kcl_gray_{S}_energy"].view(np.uint32))


@pytest.mark.parametrize("name", NAMES)
def test_driver_restatement_matches_golden(name, oracle_mod):
    """The restated GPU-branch driver on the C restatement reproduces the run made
    on the reference's own kernels."""
    O = oracle_mod
    d = load_golden(name)
    W, spin = d["W"], int(d["is_spin_glass"])
    n = W.shape[0]
    if n > 160:
        pytest.skip("O(n^3) double-flip passes: covered by the smaller instances on CPU")
    th, me = O.spin_glass_gpu_path(W, d["best_guess"], spin, int(d["e2e_gray_iterations"]), 148, 148)
    assert np.array_equal(th, d["e2e_theta"])
    assert me == pytest.approx(float(d["e2e_max_energy"]), rel=1e-12, abs=1e-9)


def test_exact_fixtures(oracle_mod):
    import itertools

    from pyqrackising_b200 import util

    d = load_golden("exact")
    assert util.int_to_bitstring(37, 8) == str(d["int_to_bitstring_37_8"])
    for n in (5, 12):
        W = d[f"W_{n}"]
        best_c, best_s = -1.0, -1.0
        mc = ms = 0
        for mask in range(1 << n):
            bits = [(mask >> i) & 1 for i in range(n)]
            c = s = 0.0
            for i, j in itertools.combinations(range(n), 2):
                if bits[i] != bits[j]:
                    c += float(W[i, j])
                s += float(W[i, j]) if bits[i] == bits[j] else -float(W[i, j])
            if c > best_c:
                best_c, mc = c, mask
            if s > best_s:
                best_s, ms = s, mask
        assert best_c == float(d[f"maxcut_value_{n}"])
        assert best_s == float(d[f"spin_value_{n}"])
        assert np.array_equal(np.array([(mc >> i) & 1 for i in range(n)], bool), d[f"maxcut_bits_{n}"])
        assert np.array_equal(np.array([(ms >> i) & 1 for i in range(n)], bool), d[f"spin_bits_{n}"])
