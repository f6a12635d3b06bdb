"""Batched local search (pqi_batch_search): many graphs of uneven size and many
starting states in one launch, checked against the oracle's steepest ascent and
float64 re-scoring."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _graphs(kind, sizes, seed=0):
    from pyqrackising_b200 import workloads as wl

    out = []
    for i, n in enumerate(sizes):
        if kind == "int":
            W = wl.regular_pm1_fast(n + (n % 2), seed=seed + i)
        else:
            W = wl.gnp_weighted(n, 0.1, seed=seed + i, dist="uniform")
        out.append(W)
    return out


@pytest.mark.parametrize("kind", ["int", "float"])
def test_ascent_matches_oracle_on_uneven_batch(kind, oracle_mod):
    from pyqrackising_b200.batch import BatchedSearch
    from pyqrackising_b200.device import DeviceGraph

    O = oracle_mod
    Ws = _graphs(kind, [64, 100, 257, 190, 1000], seed=3)
    dgs = [DeviceGraph(W) for W in Ws]
    bs = BatchedSearch(dgs)
    rng = np.random.default_rng(1)
    task_graph = [0, 1, 2, 3, 4, 4, 2, 0]
    states = [rng.random(Ws[g].shape[0]) < 0.5 for g in task_graph]
    words = bs.pack_states(task_graph, states)
    for spin in (0, 1):
        vals, best, flips, status = bs.run(task_graph, words, spin, rounds=0)
        assert int(status.item()) == 0
        got = bs.unpack(best, task_graph)
        total = 0
        for t, g in enumerate(task_graph):
            ref, nf = O.steepest_ascent(Ws[g], states[t])
            total += nf
            assert np.array_equal(got[t], ref), (t, g)
            exact = O.compute_energy(got[t], Ws[g]) if spin else O.compute_cut(got[t], Ws[g])
            assert float(vals[t]) == pytest.approx(exact, rel=1e-9, abs=1e-6)
        assert int(flips.item()) == total


def test_iterated_search_improves_and_is_deterministic(oracle_mod):
    from pyqrackising_b200.batch import BatchedSearch
    from pyqrackising_b200.device import DeviceGraph
    from pyqrackising_b200 import workloads as wl

    O = oracle_mod
    W = wl.sherrington_kirkpatrick(512, seed=2)
    bs = BatchedSearch([DeviceGraph(W)])
    task_graph = [0] * 64
    words = bs.random_states(task_graph, seed=9)
    v0, _, _, _ = bs.run(task_graph, words, 1, rounds=0)
    # kicks of n/16 forced flips: small kicks are undone by the next ascent
    v1, best1, _, _ = bs.run(task_graph, words, 1, rounds=20, kick=32, seed=4)
    v2, best2, _, _ = bs.run(task_graph, words, 1, rounds=20, kick=32, seed=4)
    assert torch.equal(v1, v2) and torch.equal(best1, best2)
    assert torch.all(v1 >= v0 - 1e-9)
    assert float(v1.max()) > float(v0.max())
    states = bs.unpack(best1, task_graph)
    for t in range(0, 64, 16):
        assert float(v1[t]) == pytest.approx(O.compute_energy(states[t], W), rel=1e-9, abs=1e-6)


def test_proposal_distribution_kicks():
    """Kicks drawn from a proposal CDF: a distribution on one node flips only it."""
    from pyqrackising_b200.batch import BatchedSearch
    from pyqrackising_b200.device import DeviceGraph
    from pyqrackising_b200 import workloads as wl

    W = wl.regular_pm1_fast(128, seed=1)
    bs = BatchedSearch([DeviceGraph(W)])
    task_graph = [0] * 8
    words = bs.random_states(task_graph, seed=1)
    cdf = torch.zeros(128, dtype=torch.float64, device="cuda")
    cdf[37:] = 1.0  # all mass on node 37
    off = torch.zeros(1, dtype=torch.int64, device="cuda")
    v, _, flips, status = bs.run(task_graph, words, 1, rounds=3, kick=1, seed=2, kick_cdf=cdf, cdf_offset=off)
    v0, _, _, _ = bs.run(task_graph, words, 1, rounds=0)
    assert int(status.item()) == 0
    assert torch.all(v >= v0)


@pytest.mark.parametrize("kind", ["int", "float"])
@pytest.mark.parametrize("csize", [2, 8, 16])
def test_cluster_ascent_matches_oracle(kind, csize, oracle_mod):
    """One thread-block cluster per task: the same states, values and flip
    counts as the oracle's steepest ascent (and hence as the batched kernel),
    on uneven graphs including sizes that leave CTAs of a cluster idle."""
    from pyqrackising_b200.batch import BatchedSearch
    from pyqrackising_b200.device import DeviceGraph

    O = oracle_mod
    Ws = _graphs(kind, [64, 100, 257, 190, 1000, 3000], seed=5)
    dgs = [DeviceGraph(W) for W in Ws]
    bs = BatchedSearch(dgs)
    rng = np.random.default_rng(2)
    task_graph = [5, 0, 1, 2, 3, 4, 4, 2, 0, 5]
    states = [rng.random(Ws[g].shape[0]) < 0.5 for g in task_graph]
    words = bs.pack_states(task_graph, states)
    for spin in (0, 1):
        vals, best, flips, status = bs.cluster_ascent(task_graph, words, spin, cluster_size=csize)
        assert int(status.item()) == 0
        got = bs.unpack(best, task_graph)
        total = 0
        for t, g in enumerate(task_graph):
            ref, nf = O.steepest_ascent(Ws[g], states[t])
            total += nf
            assert np.array_equal(got[t], ref), (t, g)
            exact = O.compute_energy(got[t], Ws[g]) if spin else O.compute_cut(got[t], Ws[g])
            assert float(vals[t]) == pytest.approx(exact, rel=1e-9, abs=1e-6)
        assert int(flips.item()) == total
        bvals, bbest, bflips, _ = bs.run(task_graph, words, spin, rounds=0)
        assert torch.equal(bbest, best)
        assert int(bflips.item()) == int(flips.item())


def test_cluster_ascent_flip_budget_reports_timeout():
    from pyqrackising_b200.batch import BatchedSearch
    from pyqrackising_b200.device import DeviceGraph
    from pyqrackising_b200 import workloads as wl

    W = wl.sherrington_kirkpatrick(2048, seed=4)
    bs = BatchedSearch([DeviceGraph(W)])
    words = bs.random_states([0, 0], seed=3)
    vals, best, flips, status = bs.cluster_ascent([0, 0], words, 1, cluster_size=4, flip_budget=5)
    assert int(status.item()) == 3  # PQI_ETIMEOUT
    bvals, bbest, bflips, bstatus = bs.run([0, 0], words, 1, rounds=0, flip_budget=5)
    assert int(bstatus.item()) == 3
    assert torch.equal(bbest, best)
    assert int(flips.item()) == int(bflips.item()) == 10
    assert torch.allclose(vals, bvals, rtol=1e-12, atol=1e-9)


def test_cluster_ascent_target_mode(oracle_mod):
    """Target mode: a target no task reaches leaves every result as the plain
    run's (the 16-flip checks do not change the trajectory); a target the
    best task reaches mid-ascent ends the launch early, with that task at or
    above the target and each value equal to its state's exact value."""
    from pyqrackising_b200.batch import BatchedSearch
    from pyqrackising_b200.device import DeviceGraph
    from pyqrackising_b200 import workloads as wl

    O = oracle_mod
    W = wl.sherrington_kirkpatrick(2048, seed=6)
    bs = BatchedSearch([DeviceGraph(W)])
    tasks = [0] * 12
    words = bs.random_states(tasks, seed=5)
    v0, b0, f0, s0 = bs.cluster_ascent(tasks, words, 1, cluster_size=8)
    v1, b1, f1, s1 = bs.cluster_ascent(tasks, words, 1, cluster_size=8, target=1e300)
    assert int(s0.item()) == int(s1.item()) == 0
    assert torch.equal(b0, b1) and torch.equal(v0, v1) and int(f0.item()) == int(f1.item())
    # a value every start passes well before its end: the launch stops early
    target = 0.9 * float(v0.min())
    v2, b2, f2, s2 = bs.cluster_ascent(tasks, words, 1, cluster_size=8, target=target)
    assert int(s2.item()) == 0
    assert float(v2.max()) >= target
    assert int(f2.item()) < int(f0.item())
    states = bs.unpack(b2, tasks)
    for t in range(len(tasks)):
        assert float(v2[t]) == pytest.approx(O.compute_energy(states[t], W), rel=1e-9, abs=1e-6)


@pytest.mark.parametrize("kind", ["int", "float"])
def test_warp_form_matches_cta_form(kind):
    """One warp per task gives the CTA form's best states, values and flip
    counts, with rounds of uniform and proposal-drawn kicks, on uneven sizes
    that cover every register-group count (n <= 128, 256, 512, 1024)."""
    from pyqrackising_b200.batch import BatchedSearch
    from pyqrackising_b200.device import DeviceGraph

    Ws = _graphs(kind, [40, 100, 129, 250, 300, 513, 777, 1024], seed=11)
    bs = BatchedSearch([DeviceGraph(W) for W in Ws])
    task_graph = [g for g in range(len(Ws)) for _ in range(5)]
    words = bs.random_states(task_graph, seed=9)
    # a proposal distribution per graph (normalised cumulative sums)
    rng = np.random.default_rng(4)
    cdfs, offs, off = [], [], 0
    for W in Ws:
        p = rng.random(W.shape[0]) + 0.05
        c = np.cumsum(p / p.sum())
        c[-1] = 1.0
        cdfs.append(c)
        offs.append(off)
        off += len(c)
    cdf = torch.from_numpy(np.concatenate(cdfs)).cuda()
    off_t = torch.tensor(offs, dtype=torch.int64).cuda()
    for spin in (0, 1):
        for rounds, kick, use_cdf in ((0, 0, False), (3, 8, False), (2, 5, True)):
            kw = dict(rounds=rounds, kick=kick, seed=123, kick_cdf=cdf if use_cdf else None,
                      cdf_offset=off_t if use_cdf else None)
            v1, b1, f1, s1 = bs.run(task_graph, words, spin, variant="cta", **kw)
            v2, b2, f2, s2 = bs.run(task_graph, words, spin, variant="warp", **kw)
            assert int(s1.item()) == int(s2.item()) == 0
            assert torch.equal(b1, b2), (spin, rounds, kick, use_cdf)
            assert int(f1.item()) == int(f2.item())
            if kind == "int":
                assert torch.equal(v1, v2)
            else:
                assert torch.allclose(v1, v2, rtol=1e-12, atol=1e-9)


def test_batched_solver_mixed_kinds_graph_capture(oracle_mod):
    """Mixed int8/float graphs, several seeds each: autotuned forms, one CUDA
    graph per step; per-graph results equal the best of a direct run and are
    local optima whose values match float64 re-scoring."""
    from pyqrackising_b200 import workloads as wl
    from pyqrackising_b200.batch import BatchedSearch, BatchedSolver
    from pyqrackising_b200.device import DeviceGraph

    O = oracle_mod
    Ws = wl.batched_uneven(8, lo=64, hi=300, seed=3)
    dgs = [DeviceGraph(W) for W in Ws]
    solver = BatchedSolver(dgs, seeds_per_graph=6, is_spin_glass=True, rounds=2, kick=6, seed=5)
    tuning = solver.autotune(sample_tasks=24, reps=1)
    assert tuning and all(len(v) >= 2 for v in tuning.values())
    solver.set_starts(seed=17)
    solver.capture()
    solver.step()
    torch.cuda.synchronize()
    values, states, flips, status = solver.results()
    assert status == 0 and flips > 0
    for gi, W in enumerate(Ws):
        n = W.shape[0]
        bits = np.unpackbits(states[gi].cpu().numpy().view(np.uint8), bitorder="little")[:n].astype(bool)
        assert float(values[gi]) == pytest.approx(O.compute_energy(bits, W), rel=1e-9, abs=1e-6)
        x = np.where(bits, 1.0, -1.0)
        Wd = W.astype(np.float64).copy()
        np.fill_diagonal(Wd, 0.0)
        assert np.all(x * (Wd @ x) <= 1e-6 * np.abs(Wd).sum(axis=1).max())  # local optimum
    # the replay equals a direct run of the same group
    grp = solver.groups[0]
    form, wps = grp["form"]
    v2, _, _, _ = grp["bs"].run(grp["tg"], grp["init"], True, rounds=2, kick=6, seed=5, variant=form, warps_per_sm=wps)
    assert torch.allclose(v2, grp["out"][1], rtol=0, atol=0)


@pytest.mark.parametrize("kind", ["int", "float"])
def test_float32_fields_form(kind, oracle_mod):
    """fields="f32": int8 graphs are unchanged (exact int32 fields); float
    graphs end at local optima whose returned values match float64
    re-scoring within float32-gain accuracy."""
    from pyqrackising_b200.batch import BatchedSearch
    from pyqrackising_b200.device import DeviceGraph

    O = oracle_mod
    Ws = _graphs(kind, [100, 257, 1000, 2500], seed=8)
    bs = BatchedSearch([DeviceGraph(W) for W in Ws])
    task_graph = [0, 1, 2, 3, 3, 2]
    words = bs.random_states(task_graph, seed=4)
    v64, b64, f64, _ = bs.run(task_graph, words, True, rounds=2, kick=6, seed=3)
    v32, b32, f32, st = bs.run(task_graph, words, True, rounds=2, kick=6, seed=3, fields="f32")
    assert int(st.item()) == 0
    if kind == "int":
        assert torch.equal(b32, b64) and torch.equal(v32, v64)
        return
    for t, g in enumerate(task_graph):
        bits = bs.unpack(b32, task_graph)[t]
        W = Ws[g]
        e = O.compute_energy(bits, W)
        assert float(v32[t]) == pytest.approx(e, rel=1e-5, abs=1e-5 * np.abs(W).sum())
        x = np.where(bits, 1.0, -1.0)
        Wd = W.astype(np.float64).copy()
        np.fill_diagonal(Wd, 0.0)
        assert np.all(x * (Wd @ x) <= 1e-5 * np.abs(Wd).sum(axis=1).max())


def test_float32_fields_staged_rows_match_register_rows():
    """Graphs above 4096 nodes (one with a ragged last group): the float32
    form with four row groups per thread staged through cp.async returns the
    same states, values and flip counts as with every group in registers, and
    its states are local optima of the float64 objective."""
    from pyqrackising_b200 import _lib
    from pyqrackising_b200 import workloads as wl
    from pyqrackising_b200.batch import BatchedSearch
    from pyqrackising_b200.device import DeviceGraph

    Ws = [wl.gnp_weighted(4099, 0.2, seed=21, dist="normal"), wl.gnp_weighted(9001, 0.05, seed=22, dist="normal")]
    bs = BatchedSearch([DeviceGraph(W) for W in Ws])
    task_graph = [0, 1, 1, 0, 1]
    words = bs.random_states(task_graph, seed=6)
    try:
        _lib.call("pqi_batch_set_staging", 0)
        va, ba, fa, sa = bs.run(task_graph, words, True, rounds=1, kick=8, seed=2, fields="f32")
        _lib.call("pqi_batch_set_staging", 1)
        vb, bb, fb, sb = bs.run(task_graph, words, True, rounds=1, kick=8, seed=2, fields="f32")
    finally:
        _lib.call("pqi_batch_set_staging", 1)
    assert int(sa.item()) == 0 and int(sb.item()) == 0
    assert torch.equal(ba, bb) and torch.equal(va, vb) and int(fa.item()) == int(fb.item())
    for t, g in enumerate(task_graph):
        bits = bs.unpack(bb, task_graph)[t]
        W = Ws[g].astype(np.float64)
        np.fill_diagonal(W, 0.0)
        x = np.where(bits, 1.0, -1.0)
        assert float(vb[t]) == pytest.approx(-0.5 * x @ W @ x, rel=1e-5)
        assert np.all(x * (W @ x) <= 1e-5 * np.abs(W).sum(axis=1).max())


@pytest.mark.parametrize("sizes", [(8192, 5000, 4500), (12000, 9000, 8300)])
def test_tmem_fields_match_shared_memory_fields(sizes):
    """Float64 fields in tensor memory (float graphs of 4097-8192 nodes, four
    tasks per SM; 8193-16384 nodes, two) give the same states, values and flip
    counts as the fields in shared memory, for dense graphs (starting fields
    from the start pass) and row-list graphs (summed by each field's owner),
    with kicks; the values are the float64 objective of the states."""
    from pyqrackising_b200 import _lib
    from pyqrackising_b200 import workloads as wl
    from pyqrackising_b200.batch import BatchedSearch
    from pyqrackising_b200.device import DeviceGraph

    n0, n1, n2 = sizes
    Ws = [wl.sherrington_kirkpatrick(n0, seed=31), wl.gnp_weighted(n1, 0.02, seed=32, dist="normal"),
          wl.gnp_weighted(n2, 0.3, seed=33, dist="uniform")]
    bs = BatchedSearch([DeviceGraph(W) for W in Ws])
    task_graph = [0, 1, 2, 0, 1, 2, 0]
    words = bs.random_states(task_graph, seed=8)
    try:
        _lib.call("pqi_batch_set_tmem_fields", 0)
        va, ba, fa, sa = bs.run(task_graph, words, True, rounds=2, kick=6, seed=4)
        _lib.call("pqi_batch_set_tmem_fields", 1)
        vb, bb, fb, sb = bs.run(task_graph, words, True, rounds=2, kick=6, seed=4)
    finally:
        _lib.call("pqi_batch_set_tmem_fields", 1)
    assert int(sa.item()) == 0 and int(sb.item()) == 0
    assert torch.equal(ba, bb) and torch.equal(va, vb) and int(fa.item()) == int(fb.item())
    for t, g in enumerate(task_graph[:3]):
        bits = bs.unpack(bb, task_graph)[t]
        W = Ws[g].astype(np.float64)
        np.fill_diagonal(W, 0.0)
        x = np.where(bits, 1.0, -1.0)
        assert float(vb[t]) == pytest.approx(-0.5 * x @ W @ x, rel=1e-9)


@pytest.mark.parametrize("kind", ["int", "float"])
def test_cta128_form_matches_cta_form(kind):
    """The 128-thread CTA form (pqi_batch_search_cta) follows the 256-thread
    form exactly: same fields summed in the same order, same selection and
    kick stream, so the same states, values and flip counts, for float64 and
    float32 fields."""
    from pyqrackising_b200.batch import BatchedSearch
    from pyqrackising_b200.device import DeviceGraph

    Ws = _graphs(kind, [64, 130, 257, 700, 1000, 2500], seed=12)
    bs = BatchedSearch([DeviceGraph(W) for W in Ws])
    task_graph = [0, 1, 2, 3, 4, 5, 4, 3, 1]
    words = bs.random_states(task_graph, seed=8)
    for fields in ("f64", "f32"):
        a = bs.run(task_graph, words, True, rounds=2, kick=5, seed=4, fields=fields)
        for variant in ("cta128", "cta64"):
            b = bs.run(task_graph, words, True, rounds=2, kick=5, seed=4, fields=fields, variant=variant)
            assert int(a[3].item()) == 0 and int(b[3].item()) == 0
            assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1]) and int(a[2].item()) == int(b[2].item())


def test_row_list_starts_match_dense_starts():
    """Starting fields from row lists (sparse graphs) against the dense row
    reads: int8 graphs give identical searches (exact sums); float graphs of
    2048+ nodes too (both sum each field in column order); smaller float
    graphs (the dense start reduces by warp shuffles) end at local optima with
    values equal to float64 re-scoring."""
    from pyqrackising_b200.batch import BatchedSearch
    from pyqrackising_b200.device import DeviceGraph

    for kind, sizes, exact in (("int", [64, 300, 1000, 2100], True), ("float", [2100, 2600], True),
                               ("float", [100, 700], False)):
        Ws = _graphs(kind, sizes, seed=30)
        dgs = [DeviceGraph(W) for W in Ws]
        with_lists = BatchedSearch(dgs)
        dense = BatchedSearch(dgs, row_lists=False)
        # the lists are really attached (these graphs are at most 10 % nonzero),
        # and really absent from the dense descriptors
        from pyqrackising_b200.batch import _DESC

        adj = np.frombuffer(with_lists.desc.cpu().numpy().tobytes(), dtype=_DESC)["adj_ptr"]
        assert np.all(adj != 0)
        assert np.all(np.frombuffer(dense.desc.cpu().numpy().tobytes(), dtype=_DESC)["adj_ptr"] == 0)
        task_graph = [i % len(Ws) for i in range(3 * len(Ws))]
        words = with_lists.random_states(task_graph, seed=9)
        for variant in ("cta", "cta64"):
            a = with_lists.run(task_graph, words, True, rounds=1, kick=4, seed=1, variant=variant)
            b = dense.run(task_graph, words, True, rounds=1, kick=4, seed=1, variant=variant)
            assert int(a[3].item()) == 0 and int(b[3].item()) == 0
            if exact:
                assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1]) and int(a[2].item()) == int(b[2].item())
            else:
                for t, g in enumerate(task_graph):
                    bits = with_lists.unpack(a[1], task_graph)[t]
                    W = Ws[g].astype(np.float64)
                    np.fill_diagonal(W, 0.0)
                    x = np.where(bits, 1.0, -1.0)
                    assert float(a[0][t]) == pytest.approx(-0.5 * x @ W @ x, rel=1e-9, abs=1e-9)
                    assert np.all(x * (W @ x) <= 1e-9 * np.abs(W).sum(axis=1).max())


@pytest.mark.parametrize("kind", ["int", "float"])
def test_start_pass_gives_the_per_task_fields(kind, oracle_mod):
    """The batched starting-field pass (one pass over W per tile of 64 tasks x
    64 nodes) against every task summing its own fields: dense graphs (no row
    lists), tasks of several graphs interleaved so tiles hold mixed graphs.
    Integer weights: identical searches. Float weights: above 2048 nodes the
    two sums run in the same order (identical searches); below, each value is
    its state's exact value."""
    from pyqrackising_b200 import _lib
    from pyqrackising_b200.batch import BatchedSearch
    from pyqrackising_b200.device import DeviceGraph

    O = oracle_mod
    sizes = [64, 257, 1000, 2100, 3000]
    Ws = _graphs(kind, sizes, seed=21)
    bs = BatchedSearch([DeviceGraph(W) for W in Ws], row_lists=False)
    rng = np.random.default_rng(4)
    task_graph = [int(g) for g in rng.integers(0, len(sizes), 150)]
    words = bs.random_states(task_graph, seed=8)
    for fields in (("f64", "f32") if kind == "float" else ("f64",)):
        out = {}
        for on in (1, 0):
            _lib.call("pqi_batch_set_start_pass", on)
            try:
                out[on] = bs.run(task_graph, words, 1, rounds=2, kick=4, seed=3, fields=fields)
                out[(on, "c")] = bs.cluster_ascent(task_graph, words, 1, cluster_size=4)
            finally:
                _lib.call("pqi_batch_set_start_pass", 1)
        for key in ((1, 0), ((1, "c"), (0, "c"))):
            a, b = out[key[0]], out[key[1]]
            if kind == "int":
                assert torch.equal(a[1], b[1]) and torch.equal(a[0], b[0]) and int(a[2].item()) == int(b[2].item())
                continue
            states = bs.unpack(a[1], task_graph)
            for t, g in enumerate(task_graph):
                if sizes[g] >= 2048 and fields == "f64":
                    assert float(a[0][t]) == float(b[0][t])
                if t % 10 == 0:
                    assert float(a[0][t]) == pytest.approx(O.compute_energy(states[t], Ws[g]), rel=1e-9, abs=1e-6)
