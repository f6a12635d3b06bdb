"""Kernel-level parity on the GPU: libpqi against the reference's own outputs
(golden fixtures from kernels.cl run on the host and from the reference's numba
code) and against the oracle on fresh inputs.

Tolerances: integer weights must match bit for bit (values and selected
indices). Float weights: values within 1e-5 relative to the row's absolute sum
(gains) or to the sum of |W| (cuts), the stated bound for float32 inputs;
the reference itself sums in float32, so its own error is of that order.
"""

import numpy as np
import pytest
import torch

from conftest import golden_names, load_golden

pytestmark = pytest.mark.gpu

NAMES = golden_names()


@pytest.fixture(scope="module", autouse=True)
def _device():
    from pyqrackising_b200 import _lib

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    assert _lib.load().pqi_check_device(torch.cuda.current_device()) == 0, "not an sm_100 device"
    yield


def _graph(W):
    from pyqrackising_b200.device import DeviceGraph

    return DeviceGraph(W)


def _is_int(W):
    return bool(np.all(W == np.rint(W)) and np.abs(W).max() <= 127)


@pytest.mark.parametrize("name", NAMES)
def test_prepare_pack_rescore(name, oracle_mod):
    O = oracle_mod
    d = load_golden(name)
    W, th = d["W"], d["theta"]
    dg = _graph(W)
    assert dg.is_integer == _is_int(W)
    assert dg.upper_sum == pytest.approx(float(np.triu(W.astype(np.float64), 1).sum()), rel=1e-12, abs=1e-9)
    words = dg.pack(th)
    got = words[: dg.n32].cpu().numpy().view(np.uint32)
    assert np.array_equal(got, d["ref_convert_bool_to_uint"])
    assert np.array_equal(dg.unpack(words)[0], th)
    cut, en = dg.rescore(words)
    assert float(cut.item()) == pytest.approx(O.compute_cut(th, W), rel=1e-12, abs=1e-9)
    assert float(en.item()) == pytest.approx(O.compute_energy(th, W), rel=1e-12, abs=1e-9)


@pytest.mark.parametrize("name", NAMES)
def test_gains_and_single_flips(name, oracle_mod):
    O = oracle_mod
    d = load_golden(name)
    W, th, spin = d["W"], d["theta"], int(d["is_spin_glass"])
    n = W.shape[0]
    dg = _graph(W)
    words = dg.pack(th)
    g32, g64 = dg.gains(words)
    ref = d["ref_cut_diff"]
    if _is_int(W):
        assert np.array_equal(g64.cpu().numpy(), ref)
        assert np.array_equal(g32.cpu().numpy(), ref.astype(np.float32))
    else:
        tol = 1e-5 * np.abs(W.astype(np.float64)).sum(axis=1) + 1e-7
        assert np.all(np.abs(g64.cpu().numpy() - ref) <= tol)
    for mpe in (148, 4096):
        G, L = O.flip_geometry(n, mpe)
        be, bi = dg.single_bit_flips(words, spin, G, L)
        ke, ki = d[f"kcl_single_{mpe}"]
        if _is_int(W):
            assert (float(be.item()), int(bi.item())) == (float(np.float32(ke)), int(ki))
        else:
            assert float(be.item()) == pytest.approx(float(ke), rel=1e-5, abs=1e-5)
            assert int(bi.item()) == int(ki)


@pytest.mark.parametrize("name", NAMES)
def test_double_flips(name, oracle_mod):
    O = oracle_mod
    d = load_golden(name)
    W, th, spin = d["W"], d["theta"], int(d["is_spin_glass"])
    n = W.shape[0]
    dg = _graph(W)
    words = dg.pack(th)
    _, g64 = dg.gains(words)
    for mpe in (148, 4096):
        G, L = O.flip_geometry(n, mpe)
        for gains in (g64, None):
            be, bi = dg.double_bit_flips(words, gains, spin, G, L)
            ke, kc = d[f"kcl_double_{mpe}"]
            if _is_int(W):
                assert (float(be.item()), int(bi.item())) == (float(np.float32(ke)), int(kc))
            else:
                assert float(be.item()) == pytest.approx(float(ke), rel=1e-5, abs=1e-5)
                assert int(bi.item()) == int(kc)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("path", [0, 1, 2, 5])
def test_calculate_cut(name, path, oracle_mod):
    from pyqrackising_b200 import _lib

    O = oracle_mod
    d = load_golden(name)
    W, spin = d["W"], int(d["is_spin_glass"])
    X = d["cut_candidates"]
    shots = X.shape[0]
    dg = _graph(W)
    words = dg.pack(X)
    G, L = O.cut_geometry(shots, 148)
    _lib.call("pqi_score_set_path", path)
    try:
        e, be, bi = dg.calculate_cut(words, shots, spin, G, L)
    finally:
        _lib.call("pqi_score_set_path", 0)
    ref_vals = O.cut_values(W, O.pack32(X), shots, spin)
    ke, ki = d["kcl_cut_148"]
    if _is_int(W):
        assert np.array_equal(e.cpu().numpy(), ref_vals)
        assert (float(be.item()), int(bi.item())) == (float(np.float32(ke)), int(ki))
    else:
        exact = np.array([
            (O.compute_energy(x, W) if spin else O.compute_cut(x, W)) for x in X
        ])
        tol = 1e-5 * np.abs(W.astype(np.float64)).sum() / 2
        assert np.all(np.abs(e.cpu().numpy().astype(np.float64) - exact) <= tol)
        assert int(bi.item()) == int(np.argmax(exact))


@pytest.mark.parametrize("name", NAMES)
def test_gray(name, oracle_mod):
    d = load_golden(name)
    W, th, spin = d["W"], d["theta"], int(d["is_spin_glass"])
    dg = _graph(W)
    words = dg.pack(th)
    _, g64 = dg.gains(words)
    for S in (148, 512):
        T = int(d[f"kcl_gray_{S}_T"])
        tout, eout = dg.gray(words, g64, spin, T, S)
        t = tout.cpu().numpy().view(np.uint64).reshape(S, -1)
        e = eout.cpu().numpy()
        if _is_int(W):
            assert np.array_equal(t, d[f"kcl_gray_{S}_theta"])
            assert np.array_equal(e, d[f"kcl_gray_{S}_energy"])
        else:
            tol = 1e-5 * np.abs(W.astype(np.float64)).sum() / 2
            assert np.all(np.abs(e - d[f"kcl_gray_{S}_energy"]) <= tol)
            # a seed may end elsewhere than the reference's only if its walk
            # made a keep-or-revert decision on a gain within float32 rounding
            # of zero (the oracle reproduces the reference's walk and reports
            # each seed's smallest |gain|)
            same = np.all(t == d[f"kcl_gray_{S}_theta"], axis=1)
            rt, _, _, margin = oracle_mod.gray(W, oracle_mod.pack64(th), spin, T, S, margins=True)
            assert np.array_equal(rt, d[f"kcl_gray_{S}_theta"])
            row_scale = float(np.abs(W.astype(np.float64)).sum(axis=1).mean())
            assert np.all(same | (margin <= 1e-5 * row_scale))


def test_descent_matches_repeated_single_passes(oracle_mod):
    """pqi_single_descent == the reference's loop of single_bit_flips + flip, with
    heavy ties (+-1 weights)."""
    from pyqrackising_b200 import workloads as wl

    O = oracle_mod
    for n, seed in ((64, 42), (200, 5), (333, 9)):
        W = wl.regular_pm1(n, seed=seed) if n % 2 == 0 else wl.gnp_weighted(n, 0.2, seed=seed)
        W = np.sign(W).astype(np.float32)
        for spin in (0, 1):
            th = np.random.default_rng(seed).random(n) < 0.5
            G, L = O.flip_geometry(n, 148)
            # oracle
            ref_trace, cur, esum = [], th.copy(), 0.0
            while True:
                e, i = O.single_select(W, O.pack32(cur), spin, G, L)
                if not e > 0:
                    break
                ref_trace.append(i)
                esum += float(e)
                cur[i] = not cur[i]
            dg = _graph(W)
            words = dg.pack(th)
            _, g64 = dg.gains(words)
            trace = torch.empty(4 * n, dtype=torch.int32, device="cuda")
            es, fl, rc = dg.single_descent(words, g64, spin, G, L, 4 * n, trace)
            assert rc == 0
            assert trace[: int(fl.item())].tolist() == ref_trace
            assert float(es.item()) == esum
            assert np.array_equal(dg.unpack(words)[0], cur)
            # maintained gains equal fresh gains
            _, g_fresh = dg.gains(words)
            assert torch.equal(g64, g_fresh)


def test_exact_search_fixtures():
    from pyqrackising_b200.maxcut_tfim import exact_search

    d = load_golden("exact")
    for n in (5, 12, 20):
        W = d[f"W_{n}"]
        bits, v = exact_search(W, False)
        assert v == float(d[f"maxcut_value_{n}"]) and np.array_equal(bits, d[f"maxcut_bits_{n}"])
        bits, v = exact_search(W, True)
        assert v == float(d[f"spin_value_{n}"]) and np.array_equal(bits, d[f"spin_bits_{n}"])


def test_errors_are_reported_and_context_survives():
    from pyqrackising_b200 import _lib
    from pyqrackising_b200.device import DeviceGraph

    W = np.zeros((40, 40), np.float32)
    W[0, 1] = W[1, 0] = np.nan
    with pytest.raises(ValueError):
        DeviceGraph(W)
    W = np.zeros((40, 40), np.float32)
    W[0, 1] = 1.0
    with pytest.raises(ValueError):
        DeviceGraph(W)
    W[1, 0] = 1.0
    dg = DeviceGraph(W)
    words = dg.pack(np.zeros(40, bool))
    with pytest.raises(_lib.PQIError) as ei:
        dg.single_bit_flips(words, 0, 10, 3)  # 3 does not divide 10
    assert ei.value.status == _lib.PQI_EINVAL
    # a descent whose flip budget runs out returns PQI_ETIMEOUT, and the device stays usable
    _, g64 = dg.gains(words)
    _, fl, rc = dg.single_descent(words, g64, 0, 64, 32, 0)
    assert rc == _lib.PQI_ETIMEOUT and int(fl.item()) == 0
    cut, _ = dg.rescore(words)
    assert float(cut.item()) == 0.0
    torch.cuda.synchronize()


@pytest.mark.parametrize("n", [2, 3, 17, 100, 1023, 1025, 4097])
@pytest.mark.parametrize("kind", ["int", "float"])
def test_double_flips_odd_sizes(n, kind, oracle_mod):
    """The double pass at sizes that leave partial row groups, partial column
    chunks and fewer tiles than CTAs (each CTA streams one contiguous run of
    tiles): its selection against the reference's fold over every pair value
    float(g_k + g_l -/+ 2 W_kl), taken in float64 from the device's own gains,
    for integer (int8) and float32 weights, both objectives."""
    O = oracle_mod
    rng = np.random.default_rng(1000 + n)
    if kind == "int":
        U = np.triu(rng.integers(-3, 4, size=(n, n)).astype(np.float32), 1)
    else:
        U = np.triu(rng.standard_normal((n, n)).astype(np.float32), 1)
    W = U + U.T
    th = rng.random(n) < 0.5
    dg = _graph(W)
    assert dg.is_integer == (kind == "int")
    words = dg.pack(th)
    _, g64 = dg.gains(words)
    g = g64.cpu().numpy()
    k, l = np.triu_indices(n, 1)
    vals = (g[k] + g[l]) - np.where(th[k] == th[l], 2.0, -2.0) * W[k, l].astype(np.float64)
    G, L = O.flip_geometry(n, 148)
    for spin in (0, 1):
        v32 = vals.astype(np.float32) * np.float32(2.0 if spin else 1.0)
        ke, ki = O.select(v32, G, L)
        be, bi = dg.double_bit_flips(words, g64, spin, G, L)
        assert (float(be.item()), int(bi.item())) == (float(ke), int(ki))


@pytest.mark.parametrize("mpe", [148, 4096])
def test_double_flips_wide_geometry(mpe, oracle_mod):
    """n = 2200 with integer weights (exact pair values): the pair scan's
    selection against the reference's per-work-item fold over all pairs in
    k-major order, for a table-held geometry (G = 160) and one above the table
    (G = 2208)."""
    O = oracle_mod
    n = 2200
    rng = np.random.default_rng(11)
    U = np.triu(rng.choice(np.array([-2.0, -1.0, 0.0, 1.0, 3.0], dtype=np.float32), size=(n, n)), 1)
    W = U + U.T
    th = rng.random(n) < 0.5
    dg = _graph(W)
    words = dg.pack(th)
    _, g64 = dg.gains(words)
    x = np.where(th, 1.0, -1.0)
    g = x * (W.astype(np.float64) @ x)
    assert np.array_equal(g64.cpu().numpy(), g)
    k, l = np.triu_indices(n, 1)
    vals = g[k] + g[l] - np.where(th[k] == th[l], 2.0, -2.0) * W[k, l]
    G, L = O.flip_geometry(n, mpe)
    assert (G > 2048) == (mpe == 4096)
    for spin in (0, 1):
        ke, ki = O.select((vals * (2.0 if spin else 1.0)).astype(np.float32), G, L)
        be, bi = dg.double_bit_flips(words, g64, spin, G, L)
        assert (float(be.item()), int(bi.item())) == (float(ke), int(ki))
