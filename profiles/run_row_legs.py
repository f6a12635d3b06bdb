"""Timings of the kernels and entry points that the headline bench does not
cover, each on one B200 with CUDA events on the launching stream:

  double  one double-bit-flip pass (pair scan from maintained gains,
          kernels.cl:150-231 semantics) on SK n=8192 float32 and ER n=2048 int8
  gray    one parallel Gray-code search (kernels.cl:877-978 semantics) from a
          single-flip local optimum: SK n=8192 (n^2 iterations, 148 seeds) and
          ER(1024, 0.5) (n^2/16 iterations, the reference CPU twin's setting)
  tfim    the TFIM sampler alone (3-regular n=2048 and ER n=2048, quality 6:
          65,536 shots) and maxcut_tfim end to end on ER(1024, 0.5) at quality 2
  sparse  spin_glass_solver_sparse on G(16384, 0.01) N(0,1) against the dense
          solver on the same matrix
  bnb     solve_maxcut_bnb (exact branch and bound) on 3-regular +-1 graphs,
          n = 28 and 32, from a fixed warm start, with the reference's batch cap
          of the build container (64) and with 4096 nodes per launch

Usage: python profiles/run_row_legs.py [leg ...]  (default: all legs). One JSON
line per measurement. Exits non-zero on a library error."""

import importlib
import json
import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import numpy as np  # noqa: E402
import torch  # noqa: E402

from pyqrackising_b200 import device as D  # noqa: E402
from pyqrackising_b200 import workloads as wl  # noqa: E402

MT = importlib.import_module("pyqrackising_b200.maxcut_tfim")

HBM_GBS = None
_peaks = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
if os.path.exists(_peaks):
    with open(_peaks) as f:
        HBM_GBS = float(json.load(f).get("hbm_gbs", 0.0)) or None
HBM_GBS = HBM_GBS or 6650.0

_flush = None


def flush_l2():
    """Write 256 MB (twice the L2) so the next launch starts cold."""
    global _flush
    if _flush is None:
        _flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    _flush.fill_(1)


def timed(fn, reps, flush=True):
    """Mean device time (ms) of fn() over reps launches, L2 flushed before each."""
    total = 0.0
    for _ in range(reps):
        if flush:
            flush_l2()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        total += a.elapsed_time(b)
    return total / reps


def emit(**kw):
    print(json.dumps(kw), flush=True)


def local_optimum(dg, seed, spin=True):
    """Random state taken to a single-flip local optimum with the device descent.
    The words hold ceil(n/32) + 1 int32, so they also read as ceil(n/64) 64-bit words."""
    words = dg.pack(wl.random_bits(dg.n, seed))
    _, g64 = dg.gains(words)
    Gf, Lf = D.geometry(min(D.WORK_GROUP_MULTIPLE, dg.n), dg.n, D.max_gpu_proc_elem())
    while True:
        _, _, rc = dg.single_descent(words, g64, spin, Gf, Lf, 1 << 16)
        if rc != 3:
            break
    return words, g64, Gf, Lf


def leg_double():
    for name, W, spin in (("SK n=8192 float32", wl.sherrington_kirkpatrick(8192, seed=1), True),
                          ("ER(2048, 0.5) int8", wl.erdos_renyi(2048, 0.5, seed=1), False)):
        dg = D.DeviceGraph(W)
        n = dg.n
        words, g64, Gf, Lf = local_optimum(dg, 3, spin)
        for _ in range(3):
            dg.double_bit_flips(words, g64, spin, Gf, Lf)
        ms = timed(lambda: dg.double_bit_flips(words, g64, spin, Gf, Lf), 20)
        pairs = n * (n - 1) // 2
        wbytes = pairs * (1 if dg.is_integer else 4)
        emit(leg="double", graph=name, n=n, ms_per_pass=round(ms, 4), pairs_per_s=pairs / ms * 1e3,
             w_bytes=wbytes, gbs=round(wbytes / ms / 1e6, 1),
             hbm_frac=round(wbytes / ms / 1e6 / HBM_GBS, 3), l2_flushed=True)


def leg_gray():
    mpe = D.max_gpu_proc_elem()
    for name, W, spin, iters, seeds in (
        ("SK n=8192 float32", wl.sherrington_kirkpatrick(8192, seed=1), True, 8192 * 8192, mpe),
        ("ER(1024, 0.5) float32", wl.erdos_renyi(1024, 0.5, seed=1), False, 1024 * 1024 // 16, mpe),
    ):
        dg = D.DeviceGraph(W)
        n = dg.n
        words, g64, _, _ = local_optimum(dg, 4, spin)
        bound = (iters + seeds - 1) // seeds
        for _ in range(2):
            dg.gray(words, g64, spin, bound, seeds)
        ms = timed(lambda: dg.gray(words, g64, spin, bound, seeds), 5)
        blocks = dg.n64
        positions = sum(((bound - 1 - s) // seeds + 1) * blocks for s in range(seeds) if bound > s)
        _, eout = dg.gray(words, g64, spin, bound, seeds)
        torch.cuda.synchronize()
        emit(leg="gray", graph=name, n=n, seeds=seeds, iterations=iters, ms_per_search=round(ms, 3),
             positions=positions, positions_per_s=positions / ms * 1e3,
             improving_seeds=int((eout > 0).sum().item()))


def leg_tfim():
    for name, W in (("3-regular n=2048 +-1", wl.regular_pm1_fast(2048, seed=5)),
                    ("ER(2048, 0.5)", wl.erdos_renyi(2048, 0.5, seed=1))):
        dg = D.DeviceGraph(W)
        _, _, cum = MT.hamming_cdf(dg, 6, 8.0, 8.0)
        shots = ((max(1, (2048 << 6) >> 1) + 31) >> 5) << 5
        buf = MT.sample_batch(dg, cum, shots, 5.0, 1, 0)
        for r in range(2):
            MT.sample_batch(dg, cum, shots, 5.0, 1, r, out=buf)
        ms = timed(lambda: MT.sample_batch(dg, cum, shots, 5.0, 1, 7, out=buf), 3, flush=False)
        bits = dg.unpack(buf, rows=shots)
        emit(leg="tfim_sampler", graph=name, quality=6, shots=shots, ms_per_round=round(ms, 3),
             shots_per_s=shots / ms * 1e3, mean_selected_per_shot=float(bits.sum()) / shots,
             note="W (16 MB) is L2-resident; a selected node is a picked or underflowed weight")
    W1 = wl.erdos_renyi(1024, 0.5, seed=1)
    MT.set_seed(0)
    MT.maxcut_tfim(W1, quality=2)
    runs = []
    for seed in range(5):
        MT.set_seed(seed)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, cut, _ = MT.maxcut_tfim(W1, quality=2)
        torch.cuda.synchronize()
        runs.append((time.perf_counter() - t0, cut))
    MT.set_seed(None)
    emit(leg="maxcut_tfim", graph="ER(1024, 0.5)", quality=2, wall_s=[round(t, 4) for t, _ in runs],
         cuts=[c for _, c in runs], note="host wall time per call, W upload and preparation included")


def leg_sparse():
    import scipy.sparse as sp

    from pyqrackising_b200 import spin_glass_solver, spin_glass_solver_sparse

    W = wl.gnp_weighted(16384, 0.01, seed=1, dist="normal")
    G = sp.csr_matrix(np.triu(W, 1))
    best = "".join("1" if b else "0" for b in wl.random_bits(16384, 9))
    out = {}
    for name, fn, arg in (("sparse", spin_glass_solver_sparse, G), ("dense", spin_glass_solver, W)):
        fn(arg, best_guess=best)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, cut, _, energy = fn(arg, best_guess=best)
        torch.cuda.synchronize()
        out[name] = (time.perf_counter() - t0, cut, energy)
    emit(leg="sparse", graph="G(16384, 0.01) N(0,1)", nnz_upper=int(G.nnz),
         sparse_s=round(out["sparse"][0], 3), dense_s=round(out["dense"][0], 3),
         sparse_energy=out["sparse"][2], dense_energy=out["dense"][2],
         note="same best_guess; host wall time per call, coordinate upload / W upload included")


def leg_bnb():
    import contextlib
    import io
    import re

    from pyqrackising_b200 import solve_maxcut_bnb

    warm = solve_maxcut_bnb(wl.regular_pm1_fast(12, seed=3), best_guess="0" * 12, verbose=False)
    assert warm[4]
    for n in (28, 32):
        W = wl.regular_pm1_fast(n, seed=3)
        rng = np.random.default_rng(1)
        guess = "".join("1" if b else "0" for b in rng.random(n) < 0.5)
        for cap in (64, 4096):
            buf = io.StringIO()
            t0 = time.perf_counter()
            with contextlib.redirect_stdout(buf):
                bits, cut, _, _, certified = solve_maxcut_bnb(W, best_guess=guess, verbose=True, batch_size=cap)
            dt = time.perf_counter() - t0
            m = re.search(r"Nodes explored: (\d+)\s+\|\s+Pruned: (\d+)", buf.getvalue())
            emit(leg="bnb", graph=f"3-regular n={n} +-1", batch_size=cap, wall_s=round(dt, 3), cut=cut,
                 certified=bool(certified), nodes=int(m.group(1)), pruned=int(m.group(2)),
                 nodes_per_s=round(int(m.group(1)) / dt))


LEGS = {"double": leg_double, "gray": leg_gray, "tfim": leg_tfim, "sparse": leg_sparse, "bnb": leg_bnb}

if __name__ == "__main__":
    for name in sys.argv[1:] or list(LEGS):
        LEGS[name]()
