"""The learned proposal network on the GPU: forward and gradients of the bf16
kernels against the float64 CPU oracle, training lowers the loss, and the
trained proposals are used by the batched search."""

import numpy as np
import pytest
import torch

from oracle import mpnn_oracle as M

pytestmark = pytest.mark.gpu


def _bf16(x):
    return torch.from_numpy(np.asarray(x, np.float32)).to(torch.bfloat16).to(torch.float64).numpy()


def test_forward_and_gradients_match_float64_oracle():
    from pyqrackising_b200 import learned as L
    from pyqrackising_b200.device import DeviceGraph

    rng = np.random.default_rng(1)
    n = 96
    W = rng.standard_normal((n, n)).astype(np.float32)
    W = np.triu(W, 1)
    W = (W + W.T).astype(np.float32)
    bits = rng.random(n) < 0.5
    theta = M.init_params(5)
    net = L.ProposalNet(params=theta)
    dg = DeviceGraph(W)
    ctx = L.GraphContext(dg)
    words = dg.pack(bits)
    F = ctx.features(words)
    # oracle on the same bf16-rounded parameters and inputs
    th16 = _bf16(theta)
    Ah, s = M.norm_adj(W)
    F_ref = M.features(bits, W, s)
    F_gpu = F.to(torch.float64).cpu().numpy().reshape(n, 4)
    assert np.allclose(F_gpu, _bf16(F_ref), rtol=1e-2, atol=1e-2)
    logits, cache = net.forward(ctx, F)
    # the oracle rounds to bf16 exactly where the kernels store bf16
    ref_logits, rcache = M.forward(th16, F_gpu, _bf16(Ah), q=M.bf16_round)
    lg = logits.cpu().numpy().astype(np.float64)
    assert np.abs(lg - ref_logits).max() <= 3e-2 * (np.abs(ref_logits).max() + 1e-3)
    t = np.zeros(n)
    t[[3, 17, 40, 77]] = 0.25
    net.zero_grad()
    loss, dl, _ = net.loss_grad(logits, torch.from_numpy(t.astype(np.float32)).cuda())
    net.backward(ctx, cache, dl)
    g_gpu = net.g.cpu().numpy().astype(np.float64)
    rl, rdl = M.loss_and_dlogits(ref_logits, t)
    assert float(loss.item()) == pytest.approx(rl, rel=2e-2, abs=1e-3)
    g_ref = M.backward(th16, rcache, _bf16(Ah), rdl, q=M.bf16_round)
    cos = g_gpu @ g_ref / (np.linalg.norm(g_gpu) * np.linalg.norm(g_ref))
    assert cos > 0.999, cos
    lay, _ = M.param_layout()
    for name, (o, sh) in lay.items():
        a = g_gpu[o : o + int(np.prod(sh))]
        b = g_ref[o : o + int(np.prod(sh))]
        # float32 accumulation against float64, the same bf16 roundings on both sides
        assert np.abs(a - b).max() <= 2e-2 * (np.abs(b).max() + 1e-4), name
    # and against the pure float64 model: bf16 storage costs about 1% of the gradient
    g64 = M.backward(th16, M.forward(th16, F_gpu, _bf16(Ah))[1], _bf16(Ah), rdl)
    assert g_gpu @ g64 / (np.linalg.norm(g_gpu) * np.linalg.norm(g64)) > 0.99


def test_training_lowers_loss_and_proposals_drive_kicks():
    from pyqrackising_b200 import learned as L
    from pyqrackising_b200 import workloads as wl
    from pyqrackising_b200.batch import BatchedSearch
    from pyqrackising_b200.device import DeviceGraph

    dgs = [DeviceGraph(wl.gnp_weighted(n, 0.05, seed=i, dist="normal")) for i, n in enumerate([128, 160, 200, 256] * 2)]
    ex = L.make_examples(dgs, tasks_per_graph=8, rounds=8, seed=1)
    assert len(ex) > 8
    net = L.ProposalNet(seed=0)
    hist = L.train(net, dgs, ex, epochs=6, lr=3e-3, batch=8)
    assert np.mean(hist[-3:]) < np.mean(hist[:3])
    # proposals as the kick distribution of the batched search
    dg = dgs[0]
    ctx = L.GraphContext(dg)
    bs = BatchedSearch([dg])
    tg = [0] * 16
    w0 = bs.random_states(tg, seed=2)
    vA, wA, _, _ = bs.run(tg, w0, 1, rounds=0)
    prob = net.proposal(ctx, wA[0].reshape(-1).contiguous())
    assert torch.isfinite(prob).all() and abs(float(prob.sum()) - 1.0) < 1e-3
    cdf, off = L.task_proposals(net, dg, wA[0:1].contiguous(), temperature=1.0)
    v, _, _, status = bs.run(tg, wA.reshape(-1).contiguous(), 1, rounds=4, kick=8, seed=3, kick_cdf=cdf, cdf_offset=off)
    assert int(status.item()) == 0 and torch.all(v >= vA - 1e-9)


def test_trained_proposals_beat_uniform_kicks():
    """Ablation: the same iterated search, the same starting optima, seeds and
    kick budget, with kicks drawn from the trained network's per-task
    proposals versus uniformly, on held-out graphs of both training families.
    The trained proposals give the higher mean best value on most graphs and
    on aggregate."""
    from pyqrackising_b200 import learned as L
    from pyqrackising_b200 import workloads as wl
    from pyqrackising_b200.device import DeviceGraph
    from pyqrackising_b200.train_proposals import ils_compare, train_streaming

    net = L.ProposalNet(seed=0)
    train_streaming(net, count=384, chunk=64, seed=1)
    held = [DeviceGraph(wl.gnp_weighted(n, 0.05, seed=1000 + i, dist="normal")) for i, n in enumerate([300, 400, 512])]
    held += [DeviceGraph(wl.regular_pm1_np(n, seed=2000 + i)) for i, n in enumerate([300, 400, 512])]
    gains = []
    for dg in held:
        r = ils_compare(net, dg, starts=32, rounds=8, seed=7)
        gains.append(r["learned_mean"] - r["uniform_mean"])
    print("mean-best gain per held-out graph:", [round(g, 2) for g in gains])
    assert sum(g > 0 for g in gains) >= 5
    assert sum(gains) > 0


@pytest.mark.parametrize("n", [100, 300, 1030])
def test_tensor_core_messages_match_cuda_core_messages(n):
    """The tcgen05 message products (A_hat X, forward and backward) give the
    CUDA-core GEMM's logits and gradients to float32-accumulation accuracy,
    on sizes that are not multiples of the 128-row tile or the 64-wide K step."""
    from pyqrackising_b200 import learned as L
    from pyqrackising_b200 import workloads as wl
    from pyqrackising_b200.device import DeviceGraph

    dg = DeviceGraph(wl.gnp_weighted(n, 0.1, seed=n, dist="normal"))
    ctx = L.GraphContext(dg)
    words = dg.pack(np.random.default_rng(n).random(n) < 0.5)
    F = ctx.features(words)
    tgt = torch.full((n,), 1.0 / n, dtype=torch.float32, device="cuda")
    out = {}
    for tcore in (False, True):
        net = L.ProposalNet(seed=1)
        net.tensor_cores = tcore
        logits, cache = net.forward(ctx, F)
        _, dl, _ = net.loss_grad(logits, tgt)
        net.zero_grad()
        net.backward(ctx, cache, dl)
        out[tcore] = (logits.cpu().numpy().astype(np.float64), net.g.cpu().numpy().astype(np.float64))
    (l0, g0), (l1, g1) = out[False], out[True]
    assert np.abs(l1 - l0).max() <= 2e-2 * (np.abs(l0).max() + 1e-6)
    cos = g0 @ g1 / (np.linalg.norm(g0) * np.linalg.norm(g1))
    assert cos > 0.999


def test_kick_cdf_kernel():
    """pqi_mpnn_kick_cdf against float64 numpy: softmax(logit / T) mixed with
    the uniform distribution, cumulated and normalised; a task with a
    non-finite logit is uniform."""
    import ctypes

    from pyqrackising_b200 import _lib

    rng = np.random.default_rng(3)
    # (the kernel takes T and mix as float32: use values that float32 holds exactly)
    n, tasks, T, mix = 3001, 3, 2.5, float(np.float32(0.1))
    z = rng.standard_normal((tasks, n)).astype(np.float32) * 4
    z[2, 17] = np.nan
    cdf = torch.empty(tasks * n, dtype=torch.float64, device="cuda")
    _lib.call("pqi_mpnn_kick_cdf", ctypes.c_void_p(torch.from_numpy(z).cuda().data_ptr()), n, tasks,
              ctypes.c_float(T), ctypes.c_float(mix), ctypes.c_void_p(cdf.data_ptr()), None)
    got = cdf.cpu().numpy().reshape(tasks, n)
    for t in range(tasks):
        if t == 2:
            p = np.full(n, 1.0 / n)
        else:
            e = np.exp(z[t].astype(np.float64) / T - (z[t].astype(np.float64) / T).max())
            p = (1 - mix) * e / e.sum() + mix / n
        c = np.cumsum(p)
        np.testing.assert_allclose(got[t], c / c[-1], rtol=1e-12, atol=1e-12)
        assert got[t][-1] == 1.0
