"""Generate the golden fixtures under tests/golden/ from the reference itself.

Run in a checkout that has the reference at /root/reference (read-only):

    NUMBA_CACHE_DIR=/tmp/numba_cache python tests/golden/make_golden.py

Sources of truth, per fixture key:

* ``ref_*`` keys come from the reference's numba CPU code imported unmodified
  (``pyqrackising/maxcut_tfim_util.py``, ``spin_glass_solver.py``,
  ``maxcut_tfim.py``).
* ``kcl_*`` keys come from the reference's OpenCL kernels
  (``pyqrackising/kernels.cl``) compiled for the host and run under the
  ND-range emulator (``oracle/build_ref.sh`` -> ``oracle/_ref``).
* ``e2e_*`` keys come from the restated GPU-branch driver loop
  (``oracle.spin_glass_gpu_path``) running on the ``kcl`` kernels.

The reference's TFIM sampler is unseeded (``maxcut_tfim_util.py:692,715``), so the
``best_guess`` it produced for each instance is stored as a fixture and fed to
both sides.
"""

from __future__ import annotations

import os
import sys
import zlib

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REFERENCE = os.environ.get("PQI_REFERENCE_ROOT", "/root/reference")
sys.path.insert(0, REPO)
sys.path.insert(0, REFERENCE)
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache")

from oracle import oracle as O  # noqa: E402
from pyqrackising_b200 import workloads as wl  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def ref_modules():
    import importlib

    # the package re-exports functions under the module names, so fetch the modules
    mt = importlib.import_module("pyqrackising.maxcut_tfim")
    mu = importlib.import_module("pyqrackising.maxcut_tfim_util")
    sg = importlib.import_module("pyqrackising.spin_glass_solver")

    return mu, mt, sg


def instances():
    """(name, W, is_spin_glass) tuples; small stand-ins for the five workloads."""
    yield "c1_regular64", wl.regular_pm1(64, seed=42), True
    yield "c2_er256", wl.erdos_renyi(256, 0.5, seed=1), False
    yield "c3_sk256", wl.sherrington_kirkpatrick(256, seed=1), True
    yield "c4_reg100", wl.regular_pm1_fast(100, seed=3), True
    yield "c4_gnp150", wl.gnp_weighted(150, 0.1, seed=4, dist="uniform"), False
    yield "c5_gnp192", wl.gnp_weighted(192, 0.05, seed=5, dist="normal"), True


def make_instance(name, W, spin, mu, mt, sg):
    n = W.shape[0]
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    theta = rng.random(n) < 0.5
    d = {"W": W, "is_spin_glass": np.int32(spin), "theta": theta}

    # objectives and packing, reference numba code
    d["ref_compute_cut"] = np.float64(mu.compute_cut(theta, W, n))
    d["ref_compute_energy"] = np.float64(mu.compute_energy(theta, W, n))
    d["ref_convert_bool_to_uint"] = mu.convert_bool_to_uint(theta[None, :])
    gains = np.empty(n, dtype=np.float64)
    for k in range(n):
        st = theta.copy()
        st[k] = not st[k]
        gains[k] = mu.compute_cut_diff(k, st, W, n)
    d["ref_cut_diff"] = gains  # cut delta of flipping each k (run_single_bit_flips values)
    pairs = rng.integers(0, n, size=(32, 2))
    pairs = pairs[pairs[:, 0] != pairs[:, 1]]
    d["pairs"] = pairs.astype(np.int32)
    d["ref_cut_diff_2"] = np.array(
        [mu.compute_cut_diff_2(int(k), int(l), _flip2(theta, k, l), W, n) for k, l in pairs], dtype=np.float64
    )
    seeds = np.stack([mu.gray_mutation(i, theta, 64 * (i % ((n + 63) >> 6))) for i in range(16)])
    d["ref_gray_mutation"] = seeds
    d["ref_cut_diff_between"] = np.array([mu.compute_cut_diff_between(theta, s, W, n) for s in seeds])

    # kernel-level outputs of the reference's OpenCL kernels (host-emulated)
    th32 = O.pack32(theta)
    for mpe in (148, 4096):
        G, L = O.flip_geometry(n, mpe)
        e, i, ge, gi = O.ref_single_select(W, th32, spin, G, L)
        d[f"kcl_single_{mpe}"] = np.array([e, i], dtype=np.float64)
        d[f"kcl_single_{mpe}_groups"] = np.stack([ge.astype(np.float64), gi.astype(np.float64)])
        e, c, _, _ = O.ref_double_select(W, th32, spin, G, L)
        d[f"kcl_double_{mpe}"] = np.array([e, c], dtype=np.float64)
    shots = 256
    X = np.random.default_rng(99).random((shots, n)) < 0.5
    d["cut_candidates"] = X
    G, L = O.cut_geometry(shots, 148)
    e, i, _, _ = O.ref_cut_select(W, O.pack32(X), shots, spin, G, L)
    d["kcl_cut_148"] = np.array([e, i], dtype=np.float64)
    for S in (148, 512):
        T = (n * n + S - 1) // S
        if O.gray_has_oob(n, T, S):
            T = min(T, (1 << (n & 63)) - 1)
        tout, eout = O.ref_gray(W, O.pack64(theta), spin, T, S)
        d[f"kcl_gray_{S}_T"] = np.int64(T)
        d[f"kcl_gray_{S}_theta"] = tout
        d[f"kcl_gray_{S}_energy"] = eout

    # best_guess from the reference's own sampler (unseeded), stored as the fixture
    bg = mt.maxcut_tfim(W, quality=2 if n > 64 else 6, is_spin_glass=bool(spin))[0]
    best_guess = np.array([c == "1" for c in bg], dtype=np.bool_)
    d["best_guess"] = best_guess

    # end to end: restated GPU-branch driver on the reference kernels
    S = 148
    gi = n * n
    if O.gray_has_oob(n, (gi + S - 1) // S, S):
        gi = S * ((1 << (n & 63)) - 1)
    trace = []
    th_end, me = O.spin_glass_gpu_path(W, best_guess, spin, gi, 148, S, use_ref=True, trace=trace)
    d["e2e_gray_iterations"] = np.int64(gi)
    d["e2e_theta"] = th_end
    d["e2e_max_energy"] = np.float64(me)
    d["e2e_moves"] = np.array([{"single": 0, "double": 1, "gray": 2}[t[0]] for t in trace], dtype=np.int8)
    d["e2e_cut"] = np.float64(O.compute_cut(th_end, W))
    d["e2e_energy"] = np.float64(O.compute_energy(th_end, W))

    # the reference CPU solver from the same best_guess (its returned tuple)
    bs, cut, _, en = sg.spin_glass_solver(
        W, best_guess=[bool(b) for b in best_guess], is_spin_glass=bool(spin), is_maxcut_gpu=False, gray_iterations=gi
    )
    bits = np.array([c == "1" for c in bs], dtype=np.bool_)
    d["refcpu_theta"] = bits
    d["refcpu_cut_rescored"] = np.float64(O.compute_cut(bits, W))
    d["refcpu_energy_rescored"] = np.float64(O.compute_energy(bits, W))
    return d


def _flip2(theta, k, l):
    st = theta.copy()
    st[k] = not st[k]
    st[l] = not st[l]
    return st


def exact_fixtures(mu, mt):
    """Brute-force known answers for n < 24 (maxcut_tfim.py:288-339)."""
    d = {}
    for n, seed in ((5, 1), (12, 2), (20, 3)):
        W = wl.gnp_weighted(n, 0.6, seed=seed, dist="normal")
        bm, vm = mt.exact_maxcut(W)
        bs, vs = mt.exact_spin_glass(W)
        d[f"W_{n}"] = W
        d[f"maxcut_bits_{n}"] = bm
        d[f"maxcut_value_{n}"] = np.float64(vm)
        d[f"spin_bits_{n}"] = bs
        d[f"spin_value_{n}"] = np.float64(vs)
    d["int_to_bitstring_37_8"] = np.array(mu.int_to_bitstring(37, 8))
    state = np.zeros(70, dtype=np.bool_)
    flips = [mu.gray_code_next(state, i, 64 * (i % 2)) for i in range(40)]
    d["gray_code_next_flips"] = np.array(flips, dtype=np.int64)
    d["gray_code_next_state"] = state
    return d


def tfim_fixtures(mu, mt):
    """The sampler's deterministic parts from the reference's numba code:
    init_J_and_z and maxcut_hamming_cdf (maxcut_tfim.py:189-209,
    maxcut_tfim_util.py:654-687). init_thresholds leaves one middle entry of an
    np.empty array unset; the fixture passes that entry as 0.0 (the value the
    rebuild uses), so the reference function sees a defined input. Also the
    reference's own maxcut_tfim results (unseeded) over repeated runs."""
    import importlib

    ours = importlib.import_module("pyqrackising_b200.maxcut_tfim")
    d = {}
    for name, W, spin in (("c1", wl.regular_pm1(64, seed=42), True), ("c2", wl.erdos_renyi(256, 0.5, seed=1), False)):
        n = W.shape[0]
        J_eff, degrees = mt.init_J_and_z(W, 5.0)
        d[f"{name}_W"] = W
        d[f"{name}_J_eff"] = J_eff
        d[f"{name}_degrees"] = degrees
        for q in (2, 6):
            thr = ours.init_thresholds(n)
            d[f"{name}_thresholds"] = thr.copy()
            d[f"{name}_cum_q{q}"] = mu.maxcut_hamming_cdf(thr, n, J_eff, degrees, q, 8.0, 8.0)
        runs = [mt.maxcut_tfim(W, quality=6 if n <= 64 else 2, is_spin_glass=spin) for _ in range(8)]
        bits = [np.array([c == "1" for c in r[0]]) for r in runs]
        d[f"{name}_ref_runs_cut"] = np.array([O.compute_cut(b, W) for b in bits])
        d[f"{name}_ref_runs_energy"] = np.array([O.compute_energy(b, W) for b in bits])
    return d


def main():
    if not O.ref_available():
        O.build_ref(REFERENCE)
    mu, mt, sg = ref_modules()
    if "--tfim-only" in sys.argv:
        np.savez_compressed(os.path.join(OUT, "golden_tfim.npz"), **tfim_fixtures(mu, mt))
        return
    np.savez_compressed(os.path.join(OUT, "golden_tfim.npz"), **tfim_fixtures(mu, mt))
    for name, W, spin in instances():
        d = make_instance(name, W, spin, mu, mt, sg)
        np.savez_compressed(os.path.join(OUT, f"golden_{name}.npz"), **d)
        print(name, "n=%d" % W.shape[0], "e2e cut", d["e2e_cut"], "refcpu cut", d["refcpu_cut_rescored"])
    np.savez_compressed(os.path.join(OUT, "golden_exact.npz"), **exact_fixtures(mu, mt))


if __name__ == "__main__":
    main()
