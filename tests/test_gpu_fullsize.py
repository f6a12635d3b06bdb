"""Kernel-level parity at the full sizes of the benchmark configurations.

The fixture tests (test_gpu_kernels.py) pin the kernels to the reference's own
outputs at n <= 256. The kernels change shape with n (column-order starting
fields from 2048 nodes, staged row loads above 4096, the split-bf16 scoring at
ld = 8192, pair tiles across many column chunks), so the same checks run here
at the configurations' own sizes:

* ER G(2048, 0.5) unit weights (dense unweighted MAXCUT): the whole
  65,536-candidate batch scored bit for bit, and the reference-order selection.
* Sherrington-Kirkpatrick n = 8192, J ~ N(0,1)/sqrt(n) float32: single-flip
  gains and selection (G = 160), one double-flip pass from a single-flip local
  optimum, one Gray search (148 seeds, two Gray steps each), and split-bf16
  scoring of 1,024 candidates.
* G(16384, 0.01) with N(0,1) float32 weights: gains and scoring of 256
  candidates.

Float tolerances are relative to the value, as the target states them:
|got - fp64| <= 1e-5 |fp64| for every value whose magnitude is at least the
typical row scale s = mean_k sum_v |W_kv| (below that, relative error is not
meaningful and the bound is 1e-5 s). The float64 values come from float64
BLAS on the host. The reference's own float32 sums (the oracle's restatement,
in its order) are compared with the same float64 values and their error is
printed beside ours: the reference is itself ~1e-4 relative off float64 on
these sizes, so agreement with float64 is the stricter test. Selections must
equal the reference's (integer weights) or pick a value within the tolerance
of the float64 maximum (float weights: a different pick is accepted only when
both values lie within the tolerance, i.e. a tie at float32 resolution).
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

REL = 1e-5


def _ok_float(got, exact, scale):
    """|got - exact| <= 1e-5 max(|exact|, scale), elementwise; returns (ok, worst
    relative error over values >= scale, worst error / scale)."""
    got = np.asarray(got, dtype=np.float64)
    exact = np.asarray(exact, dtype=np.float64)
    err = np.abs(got - exact)
    bound = REL * np.maximum(np.abs(exact), scale)
    big = np.abs(exact) >= scale
    rel = float((err[big] / np.abs(exact[big])).max()) if big.any() else 0.0
    return bool(np.all(err <= bound)), rel, float(err.max() / scale)


def _unpack_pm1(words_u32, n, dtype=np.float64):
    """uint32[rows, n32] -> +-1 [rows, n] (bit j of the row = node j)."""
    b = np.unpackbits(words_u32.view(np.uint8), axis=1, bitorder="little")[:, :n]
    return np.where(b.astype(bool), 1.0, -1.0).astype(dtype)


def _cut_values_fp64(W64, X, spin, S):
    q = np.einsum("bi,bi->b", X @ W64, X)
    return -q / 2 if spin else (2 * S - q) / 4


@pytest.fixture(scope="module", autouse=True)
def _device():
    from pyqrackising_b200 import _lib

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    assert _lib.load().pqi_check_device(torch.cuda.current_device()) == 0
    yield
    torch.cuda.empty_cache()


@pytest.fixture(scope="module")
def sk8192():
    from pyqrackising_b200 import workloads as wl
    from pyqrackising_b200.device import DeviceGraph

    W = wl.sherrington_kirkpatrick(8192, seed=1)
    dg = DeviceGraph(W)
    W64 = W.astype(np.float64)
    scale = float(np.abs(W64).sum(axis=1).mean())
    yield W, W64, dg, scale
    del dg
    torch.cuda.empty_cache()


def _local_optimum(dg, O, bits):
    words = dg.pack(bits)
    _, g64 = dg.gains(words)
    G, L = O.flip_geometry(dg.n, 148)
    while True:
        _, _, rc = dg.single_descent(words, g64, True, G, L, 1 << 16)
        if rc != 3:
            break
    assert rc == 0
    return words, g64


def test_er2048_full_batch_bit_exact(oracle_mod):
    """The bench's workload: all 65,536 candidates of one batch, bit for bit,
    and the reference-order (value, index)."""
    from pyqrackising_b200 import workloads as wl
    from pyqrackising_b200.device import DeviceGraph

    O = oracle_mod
    n, B = 2048, 65536
    W = wl.erdos_renyi(n, 0.5, seed=1)
    dg = DeviceGraph(W)
    assert dg.is_integer
    rng = np.random.default_rng(1000)
    words = rng.integers(0, 1 << 32, size=(B, n // 32), dtype=np.uint64).astype(np.uint32)
    wdev = torch.from_numpy(np.ascontiguousarray(words).view(np.int32).reshape(-1)).cuda()
    G, L = O.cut_geometry(B, 148)
    S = float(np.triu(W.astype(np.float64), 1).sum())
    W32 = W.astype(np.float32)
    for spin in (0, 1):
        e, be, bi = dg.calculate_cut(wdev, B, spin, G, L)
        got = e.cpu().numpy()
        exact = np.empty(B, dtype=np.float64)
        for c0 in range(0, B, 4096):
            # integers below 2^24 throughout: float32 BLAS is exact here
            X = _unpack_pm1(words[c0:c0 + 4096], n, np.float32)
            q = np.einsum("bi,bi->b", X @ W32, X).astype(np.float64)
            exact[c0:c0 + 4096] = -q / 2 if spin else (2 * S - q) / 4
        assert np.array_equal(got.astype(np.float64), exact)
        re, ri = O.select(exact.astype(np.float32), G, L)
        assert (float(be.item()), int(bi.item())) == (float(re), ri)
        # the reference's own kernel (float32 sums in its order) on a sample
        pick = np.r_[0:64, int(ri)]
        ref = O.cut_values(W, words[pick], len(pick), spin)
        assert np.array_equal(ref.astype(np.float64), exact[pick])


def test_sk8192_gains_and_single_selection(sk8192, oracle_mod):
    O = oracle_mod
    W, W64, dg, scale = sk8192
    n = W.shape[0]
    th = np.random.default_rng(3).random(n) < 0.5
    words = dg.pack(th)
    g32, g64 = dg.gains(words)
    x = np.where(th, 1.0, -1.0)
    g = x * (W64 @ x)
    ok64, rel64, _ = _ok_float(g64.cpu().numpy(), g, scale)
    ok32, rel32, _ = _ok_float(g32.cpu().numpy(), g, scale)
    ref = O.single_values(W, O.pack32(th), 1)  # the reference's float32 sums, x2 (spin glass)
    _, rel_ref, _ = _ok_float(ref / 2, g, scale)
    print(f"\nSK8192 gains: fp64 rel {rel64:.2e}, fp32 rel {rel32:.2e}; reference fp32 sums rel {rel_ref:.2e}")
    assert ok64 and ok32 and rel64 <= 1e-12
    G, L = O.flip_geometry(n, 148)
    be, bi = dg.single_bit_flips(words, 1, G, L)
    ke, ki = O.select(ref, G, L)
    b = int(bi.item())
    assert abs(float(be.item()) - 2 * g[b]) <= REL * abs(2 * g[b])
    tol = REL * max(abs(2 * g.max()), scale)
    assert b == ki or abs(2 * g[b] - 2 * g[ki]) <= tol
    assert 2 * g[b] >= 2 * g.max() - tol


def _pair_max_fp64(W64, x, g):
    """Largest exact pair value g_k + g_l - 2 x_k x_l W_kl over k < l, its
    k-major pair index, and the runner-up value."""
    n = W64.shape[0]
    cols = np.arange(n)
    top = []  # (value, k, l) of each row block's two largest pairs
    for k0 in range(0, n, 256):
        k1 = min(n, k0 + 256)
        V = g[k0:k1, None] + g[None, :] - 2.0 * np.outer(x[k0:k1], x) * W64[k0:k1]
        V[cols[None, :] <= np.arange(k0, k1)[:, None]] = -np.inf
        for _ in range(2):
            r, l = divmod(int(np.argmax(V)), n)
            top.append((float(V[r, l]), k0 + r, l))
            V[r, l] = -np.inf
    top.sort(key=lambda t: -t[0])
    v, k, l = top[0]
    return v, k * (n - 1) - k * (k - 1) // 2 + (l - k - 1), top[1][0]


def test_sk8192_double_pass(sk8192, oracle_mod):
    O = oracle_mod
    W, W64, dg, scale = sk8192
    n = W.shape[0]
    words, g64 = _local_optimum(dg, O, np.random.default_rng(4).random(n) < 0.5)
    th = dg.unpack(words)[0]
    x = np.where(th, 1.0, -1.0)
    g = x * (W64 @ x)
    gd = g64.cpu().numpy()
    ok, rel, _ = _ok_float(gd, g, scale)
    assert ok and rel <= 1e-12
    assert g.max() <= 0  # single-flip local optimum
    G, L = O.flip_geometry(n, 148)
    be, bi = dg.double_bit_flips(words, g64, 1, G, L)
    # the selection rule itself, on the device's own gains: identical
    oe, oi = O.double_select_gains(W, O.pack32(th), gd, 1, G, L)
    assert (float(be.item()), int(bi.item())) == (float(oe), oi)
    # against float64
    vmax, imax, v2 = _pair_max_fp64(W64, x, g)
    k, l = O.pair_decode(int(bi.item()), n)
    vgot = g[k] + g[l] - 2.0 * x[k] * x[l] * W64[k, l]
    tol = REL * max(abs(vmax), scale)
    print(f"\nSK8192 double: max pair {2 * vmax:.6f} (runner-up {2 * v2:.6f}), device {float(be.item()):.6f}")
    assert abs(float(be.item()) - 2 * vgot) <= REL * abs(2 * vgot) + 1e-30
    assert int(bi.item()) == imax or abs(vgot - vmax) <= tol


def test_sk8192_gray(sk8192, oracle_mod):
    """148 seeds, two Gray steps each (iterations bound 2 x 148), from a
    single-flip local optimum; n = 8192 is a multiple of 64, so no flip lands
    beyond n. A seed's final state may differ from the reference's only if its
    walk made a keep-or-revert decision on a gain within the float tolerance."""
    O = oracle_mod
    W, W64, dg, scale = sk8192
    n = W.shape[0]
    words, g64 = _local_optimum(dg, O, np.random.default_rng(5).random(n) < 0.5)
    th = dg.unpack(words)[0]
    S, T = 148, 2 * 148
    tout, eout = dg.gray(words, g64, 1, T, S)
    t = tout.cpu().numpy().view(np.uint64).reshape(S, -1)
    e = eout.cpu().numpy().astype(np.float64)
    rt, rE, oob, margin = O.gray(W, O.pack64(th), 1, T, S, margins=True)
    assert oob == 0
    same = np.all(t == rt, axis=1)
    ambiguous = margin <= REL * scale
    print(f"\nSK8192 gray: {int(same.sum())}/{S} seeds identical, {int(ambiguous.sum())} with a decision within tolerance")
    assert np.all(same | ambiguous)
    # energies: the float64 cut change of each returned state
    x0 = np.where(th, 1.0, -1.0)
    X = _unpack_pm1(t.view(np.uint32)[:, : n // 32].copy(), n)
    Ssum = float(np.triu(W64, 1).sum())
    cut0 = (2 * Ssum - x0 @ W64 @ x0) / 4
    cuts = _cut_values_fp64(W64, X, 0, Ssum)
    exact = cuts - cut0
    ok, rel, _ = _ok_float(e, exact, scale)
    _, rel_ref, _ = _ok_float(rE[same], exact[same], scale)
    print(f"SK8192 gray energies: rel {rel:.2e} (reference fp32 sums {rel_ref:.2e})")
    assert ok


def test_sk8192_float_scoring(sk8192, oracle_mod):
    """1,024 candidates: 512 perturbations of a local optimum (1-20 % of bits
    flipped: the kind of states the search scores) and 512 uniform random ones.
    The default path scores float weights as fixed-point int8 digit planes
    with exact integer sums (error: the rounding of W to 2^-S) and meets 1e-5
    relative to the value. The split-bf16 path (pqi_score_set_path(4): hi + lo
    bf16 products, float32 accumulation over K = 8192) is measured beside it:
    its float32 accumulation leaves about 3e-5 of the value, still ten times
    closer to float64 than the reference's own float32 sums; it is held to
    1e-4 relative."""
    from pyqrackising_b200 import _lib

    O = oracle_mod
    W, W64, dg, scale = sk8192
    n = W.shape[0]
    assert not dg.is_integer
    rng = np.random.default_rng(6)
    words, _ = _local_optimum(dg, O, rng.random(n) < 0.5)
    opt = dg.unpack(words)[0]
    X = np.empty((1024, n), dtype=bool)
    for i in range(512):
        X[i] = opt ^ (rng.random(n) < rng.uniform(0.01, 0.2))
    X[512:] = rng.random((512, n)) < 0.5
    wdev = dg.pack(X)
    G, L = O.cut_geometry(1024, 148)
    Xpm = np.where(X, 1.0, -1.0)
    Ssum = float(np.triu(W64, 1).sum())
    for spin in (1, 0):
        exact = _cut_values_fp64(W64, Xpm, spin, Ssum)
        ref = O.cut_values(W, O.pack32(X[:64]), 64, spin)
        _, rel_ref, abs_ref = _ok_float(ref, exact[:64], scale)
        for path, bound in ((0, REL), (4, 1e-4)):
            _lib.call("pqi_score_set_path", path)
            try:
                e, be, bi = dg.calculate_cut(wdev, 1024, spin, G, L)
            finally:
                _lib.call("pqi_score_set_path", 0)
            got = e.cpu().numpy().astype(np.float64)
            err = np.abs(got - exact)
            rel = float((err / np.maximum(np.abs(exact), scale)).max())
            print(f"\nSK8192 scoring spin={spin} path={path}: max err / max(|value|, s) {rel:.2e}; "
                  f"reference fp32 sums {float((np.abs(ref - exact[:64]) / np.maximum(np.abs(exact[:64]), scale)).max()):.2e}")
            assert rel <= bound
            b = int(bi.item())
            assert exact[b] >= exact.max() - bound * max(abs(exact.max()), scale)


def test_gnp16384_gains_and_scoring(oracle_mod):
    from pyqrackising_b200 import workloads as wl
    from pyqrackising_b200.device import DeviceGraph

    O = oracle_mod
    n = 16384
    W = wl.gnp_weighted(n, 0.01, seed=5, dist="normal")
    dg = DeviceGraph(W)
    W64 = W.astype(np.float64)
    scale = float(np.abs(W64).sum(axis=1).mean())
    rng = np.random.default_rng(7)
    th = rng.random(n) < 0.5
    words = dg.pack(th)
    _, g64 = dg.gains(words)
    x = np.where(th, 1.0, -1.0)
    g = x * (W64 @ x)
    ok, rel, _ = _ok_float(g64.cpu().numpy(), g, scale)
    assert ok and rel <= 1e-12
    words_opt, _ = _local_optimum(dg, O, th)
    opt = dg.unpack(words_opt)[0]
    X = np.empty((256, n), dtype=bool)
    for i in range(128):
        X[i] = opt ^ (rng.random(n) < rng.uniform(0.01, 0.2))
    X[128:] = rng.random((128, n)) < 0.5
    G, L = O.cut_geometry(256, 148)
    e, be, bi = dg.calculate_cut(dg.pack(X), 256, 1, G, L)
    Ssum = float(np.triu(W64, 1).sum())
    exact = _cut_values_fp64(W64, np.where(X, 1.0, -1.0), 1, Ssum)
    ok, rel, abs_s = _ok_float(e.cpu().numpy(), exact, scale)
    print(f"\nG(16384,0.01) scoring: rel {rel:.2e} (max err / s {abs_s:.2e})")
    assert ok
    b = int(bi.item())
    assert exact[b] >= exact.max() - REL * max(abs(exact.max()), scale)
    del dg
    torch.cuda.empty_cache()
