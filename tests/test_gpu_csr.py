"""The compressed-row (CSR) search path against the dense path on the same
graphs, against the reference's sparse-path values (golden_sparse.npz), and on
a graph too large to hold as a dense matrix.

Integer weights: every value, gain, selection and trajectory must equal the
dense path's bit for bit (both are exact). Float weights: gains agree to 1e-12
relative (float64 sums in different orders) and selections agree unless two
values tie at float32 resolution.
"""

import importlib
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "golden_sparse.npz")


def _graphs():
    from pyqrackising_b200 import workloads as wl

    rng = np.random.default_rng(5)
    out = []
    # integer weights in {-2..2}, several densities and ragged sizes
    for n, p in ((64, 0.1), (300, 0.05), (1000, 0.01), (2111, 0.004)):
        U = np.triu((rng.random((n, n)) < p) * rng.choice(np.array([-2, -1, 1, 2], dtype=np.float32), (n, n)), 1)
        out.append(("int", (U + U.T).astype(np.float32)))
    out.append(("int", wl.regular_pm1_fast(512, seed=3)))
    out.append(("float", wl.gnp_weighted(700, 0.02, seed=4, dist="normal")))
    return out


def _pair(W):
    from scipy.sparse import csr_matrix

    from pyqrackising_b200.device import DeviceGraph
    from pyqrackising_b200.sparse import SparseDeviceGraph

    return DeviceGraph(W), SparseDeviceGraph(csr_matrix(np.triu(W, 1)))


@pytest.mark.parametrize("case", range(6))
def test_csr_kernels_match_dense(case, oracle_mod):
    O = oracle_mod
    kind, W = _graphs()[case]
    n = W.shape[0]
    dg, sg = _pair(W)
    assert sg.nnz == int(np.count_nonzero(W)) and sg.upper_sum == pytest.approx(dg.upper_sum, rel=1e-12)
    th = np.random.default_rng(case).random(n) < 0.5
    wd, ws = dg.pack(th), sg.pack(th)
    _, gd = dg.gains(wd)
    _, gs = sg.gains(ws)
    if kind == "int":
        assert torch.equal(gd, gs)
    else:
        assert torch.allclose(gd, gs, rtol=1e-12, atol=1e-12)
    G, L = O.flip_geometry(n, 148)
    for spin in (0, 1):
        a = dg.single_bit_flips(wd, spin, G, L)
        b = sg.single_bit_flips(ws, spin, G, L)
        assert (float(a[0].item()), int(a[1].item())) == (float(b[0].item()), int(b[1].item()))
        # double pass from the dense path's own gains (same inputs on both sides)
        a = dg.double_bit_flips(wd, gd, spin, G, L)
        b = sg.double_bit_flips(ws, gd, spin, G, L)
        assert (float(a[0].item()), int(a[1].item())) == (float(b[0].item()), int(b[1].item()))
        # float64 re-scoring and candidate scoring
        X = np.random.default_rng(100 + case).random((37, n)) < 0.5
        cd, ed = dg.rescore(dg.pack(X), rows=37)
        cs, es = sg.rescore(sg.pack(X), rows=37)
        assert torch.allclose(cd, cs, rtol=1e-12, atol=1e-9) and torch.allclose(ed, es, rtol=1e-12, atol=1e-9)
        Gc, Lc = O.cut_geometry(37, 148)
        e1, be1, bi1 = dg.calculate_cut(dg.pack(X), 37, spin, Gc, Lc)
        e2, be2, bi2 = sg.calculate_cut(sg.pack(X), 37, spin, Gc, Lc)
        if kind == "int":
            assert torch.equal(e1, e2) and int(bi1.item()) == int(bi2.item())
        else:
            assert torch.allclose(e1, e2, rtol=1e-5, atol=1e-5 * np.abs(W).sum(axis=1).mean())


@pytest.mark.parametrize("case", [0, 1, 2, 4])
def test_csr_descent_gray_and_flips_match_dense(case, oracle_mod):
    """Integer weights: the device descent's flip sequence, one Gray search
    (states and energies) and applied single and double flips are identical."""
    O = oracle_mod
    _, W = _graphs()[case]
    n = W.shape[0]
    dg, sg = _pair(W)
    th = np.random.default_rng(7 + case).random(n) < 0.5
    G, L = O.flip_geometry(n, 148)
    out = []
    for g in (dg, sg):
        words = g.pack(th)
        _, g64 = g.gains(words)
        trace = torch.empty(4 * n, dtype=torch.int32, device="cuda")
        es, fl, rc = g.single_descent(words, g64, True, G, L, 4 * n, trace)
        assert rc == 0
        nf = int(fl.item())
        tout, eout = g.gray(words, g64, True, 300, 148)
        g.apply_flip(words, g64, 3, n - 2)
        _, fresh = g.gains(words)
        assert torch.equal(g64, fresh)  # maintained gains equal fresh gains
        out.append((trace[:nf].cpu(), float(es.item()), tout.cpu(), eout.cpu(), words.cpu()))
    a, b = out
    assert torch.equal(a[0], b[0]) and a[1] == b[1]
    assert torch.equal(a[2], b[2]) and torch.equal(a[3], b[3]) and torch.equal(a[4], b[4])


@pytest.mark.parametrize("case", range(6))
def test_csr_improving_double_flip(case, oracle_mod):
    """pqi_csr_improving_double_flip: the exact pass's (value, index) whenever
    that value is > 0, else a value <= 0. States: random ones (many positive
    gains: non-adjacent pairs win), single-flip local optima (every gain <= 0:
    only adjacent pairs can improve; integer weights leave many zero gains),
    and local optima with one node's gain pushed up by a flip."""
    O = oracle_mod
    kind, W = _graphs()[case]
    n = W.shape[0]
    _, sg = _pair(W)
    G, L = O.flip_geometry(n, 148)
    rng = np.random.default_rng(40 + case)
    seen_pos = seen_nonpos = 0
    for trial in range(6):
        words = sg.pack(rng.random(n) < 0.5)
        _, g64 = sg.gains(words)
        if trial >= 2:
            sg.single_descent(words, g64, True, G, L, 8 * n)
        if trial == 4:
            sg.apply_flip(words, g64, int(rng.integers(n)))
        if trial == 5:  # a local optimum of single and double flips
            for _ in range(500):
                sg.single_descent(words, g64, True, G, L, 8 * n)
                e, i = sg.double_bit_flips(words, g64, 1, G, L)
                if not float(e.item()) > 0.0:
                    break
                from pyqrackising_b200.spin_glass_solver import pair_decode

                sg.apply_flip(words, g64, *pair_decode(int(i.item()), n))
        for spin in (0, 1):
            e0, i0 = sg.double_bit_flips(words, g64, spin, G, L)
            e1, i1 = sg.double_bit_flips(words, g64, spin, G, L, improving=True)
            v0, v1 = float(e0.item()), float(e1.item())
            if v0 > 0.0:
                seen_pos += 1
                assert (v1, int(i1.item())) == (v0, int(i0.item()))
            else:
                seen_nonpos += 1
                assert v1 <= 0.0
    assert seen_pos and seen_nonpos


def test_csr_solver_equals_dense_solver(monkeypatch):
    """spin_glass_solver_sparse on compressed rows (forced) and on the dense
    expansion, same graph and best_guess: the same bit string and values."""
    from scipy.sparse import csr_matrix

    from pyqrackising_b200 import spin_glass_solver_sparse

    for case in (1, 3, 4):
        _, W = _graphs()[case]
        n = W.shape[0]
        G = csr_matrix(np.triu(W, 1))
        guess = "".join("1" if b else "0" for b in np.random.default_rng(case).random(n) < 0.5)
        res = {}
        for path in ("dense", "csr"):
            monkeypatch.setenv("PQI_SPARSE_PATH", path)
            res[path] = spin_glass_solver_sparse(G, best_guess=guess, gray_iterations=4 * n)
        assert res["dense"][0] == res["csr"][0]
        assert res["dense"][1] == pytest.approx(res["csr"][1], abs=1e-9)
        assert res["dense"][3] == pytest.approx(res["csr"][3], abs=1e-9)


def test_csr_sampler_matches_reference_values(monkeypatch):
    """The sampler's J_eff and degrees from the stored rows on compressed rows
    equal the reference's sparse-path values; maxcut_tfim_sparse on compressed
    rows equals the dense expansion's run with the same sampler seed."""
    from scipy.sparse import csr_matrix

    from pyqrackising_b200 import maxcut_tfim_sparse
    from pyqrackising_b200.sparse import SparseDeviceGraph

    MT = importlib.import_module("pyqrackising_b200.maxcut_tfim")
    z = np.load(GOLD)
    for i in range(int(z["count"])):
        U = z[f"U{i}"]
        if U.shape[0] < 3:
            continue
        sg = SparseDeviceGraph(csr_matrix(U))
        J = torch.empty(sg.n, dtype=torch.float64, device="cuda")
        deg = torch.empty(sg.n, dtype=torch.int32, device="cuda")
        sg.tfim_jz(J, deg)
        np.testing.assert_allclose(J.cpu().numpy(), z[f"J{i}"], rtol=1e-12, atol=1e-12)
        assert np.array_equal(deg.cpu().numpy(), z[f"deg{i}"])
    # same draws on both paths (integer weights: same scores)
    _, W = _graphs()[2]
    G = csr_matrix(np.triu(W, 1))
    res = {}
    for path in ("dense", "csr"):
        monkeypatch.setenv("PQI_SPARSE_PATH", path)
        MT.set_seed(11)
        try:
            res[path] = maxcut_tfim_sparse(G, quality=2)
        finally:
            MT.set_seed(None)
    assert res["dense"][0] == res["csr"][0] and res["dense"][1] == res["csr"][1]


def test_csr_objectives_match_reference_values():
    """float64 cut and energy of the reference's recorded states
    (compute_cut_sparse / compute_energy_sparse values in golden_sparse.npz)."""
    from scipy.sparse import csr_matrix

    from pyqrackising_b200.sparse import SparseDeviceGraph

    z = np.load(GOLD)
    for i in range(int(z["count"])):
        sg = SparseDeviceGraph(csr_matrix(z[f"U{i}"]))
        states = z[f"states{i}"]
        cut, en = sg.rescore(sg.pack(states), rows=len(states))
        np.testing.assert_allclose(cut.cpu().numpy(), z[f"cut{i}"], rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(en.cpu().numpy(), z[f"energy{i}"], rtol=1e-6, atol=1e-6)


def test_graph_too_large_for_the_dense_path():
    """G(200000, 1e-4) with N(0,1) weights: 160 GB as a dense float32 matrix,
    48 MB as compressed rows. spin_glass_solver_sparse selects compressed rows
    on its own and returns a single-flip local optimum whose values equal
    float64 re-scoring on the host (scipy)."""
    import scipy.sparse as sp

    from pyqrackising_b200 import spin_glass_solver_sparse
    from pyqrackising_b200.sparse import use_compressed_rows

    n = 200000
    rng = np.random.default_rng(9)
    m = int(n * (n - 1) / 2 * 1e-4)
    r = rng.integers(0, n, size=2 * m)
    c = rng.integers(0, n, size=2 * m)
    keep = r < c
    r, c = r[keep][:m], c[keep][:m]
    U = sp.coo_matrix((rng.standard_normal(len(r)).astype(np.float32), (r, c)), shape=(n, n)).tocsr()
    U.sum_duplicates()
    assert use_compressed_rows(n)
    guess = "".join("1" if b else "0" for b in rng.random(n) < 0.5)
    bits, cut, _, energy = spin_glass_solver_sparse(U, best_guess=guess)
    s = np.array([b == "1" for b in bits])
    x = np.where(s, 1.0, -1.0)
    Wsym = (U + U.T).astype(np.float64).tocsr()
    assert np.all(x * (Wsym @ x) <= 1e-9)  # no single flip improves
    upper = sp.triu(Wsym, 1).tocoo()
    differ = s[upper.row] != s[upper.col]
    assert cut == pytest.approx(float(upper.data[differ].sum()), rel=1e-9)
    assert energy == pytest.approx(-float((upper.data * np.where(differ, 1.0, -1.0)).sum()), rel=1e-9)
