"""Learned flip proposals: a small message-passing network trained on the
search's own improving moves, run and trained on the GPU by libpqi's bf16
kernels (``pqi_mpnn_*``, float32 accumulation).

Model (hidden 64, 3 message-passing layers, bf16 weights):

    A_hat = D^-1/2 W D^-1/2,  D = diag(sum_u |W_vu|)
    H0  = relu(F A0 + b0),   F_v = [x_v, g_v / s_v, s_v / mean(s), 1]
    H_l = relu([H_{l-1}, A_hat H_{l-1}] AB_l + b_l),   l = 1, 2, 3
    logit_v = H_3 c + c0,    proposal = softmax(logit)

Training signal: for a local optimum A reached by steepest ascent, the batched
iterated local search (uniform kicks) finds a better optimum B; the target is
the uniform distribution over the nodes where A and B differ (the flips that
led somewhere better). At inference each task gets the proposal of its own
local optimum, flattened by a temperature (``task_proposals``), as the kick
distribution of the batched search (``BatchedSearch.run(kick_cdf=...)``, one
graph descriptor per task); kicks are drawn without replacement within a round. The plain search stays
both the arbiter (every returned value comes from the search's own exact
bookkeeping and float64 re-scoring) and the fallback (uniform kicks).
"""

from __future__ import annotations

import ctypes
import time

import numpy as np
import torch

from . import _lib
from . import device as D

HID = 64
FEAT = 4
LAYERS = 3


def param_layout():
    shapes = [("A0", (FEAT, HID)), ("b0", (HID,))]
    for l in range(1, LAYERS + 1):
        shapes += [(f"AB{l}", (2 * HID, HID)), (f"b{l}", (HID,))]
    shapes += [("c", (HID,)), ("c0", (1,))]
    out, off = {}, 0
    for name, shp in shapes:
        size = int(np.prod(shp))
        out[name] = (off, shp)
        off += size
    return out, off


def _p(t):
    return D._ptr(t)


class GraphContext:
    """Per-graph tensors of the network: the normalised adjacency (bf16) and
    the row sums of |W|."""

    def __init__(self, dg: D.DeviceGraph):
        self.dg = dg
        n = dg.n
        self.n = n
        self.ld = ((n + 7) // 8) * 8
        self.Ah = torch.empty(n * self.ld, dtype=torch.bfloat16, device=dg.device)
        self.s = torch.empty(n, dtype=torch.float32, device=dg.device)
        _lib.call("pqi_mpnn_norm_adj", _p(dg.W), n, _p(self.Ah), self.ld, _p(self.s), dg.sp())
        total = torch.empty(1, dtype=torch.float64, device=dg.device)
        _lib.call("pqi_mpnn_sum", _p(self.s), n, _p(total), dg.sp())
        self.mean_s = float(total.item()) / n

    def features(self, words: torch.Tensor, g64: torch.Tensor | None = None) -> torch.Tensor:
        if g64 is None:
            _, g64 = self.dg.gains(words)
        F = torch.empty(self.n * FEAT, dtype=torch.bfloat16, device=self.dg.device)
        _lib.call("pqi_mpnn_features", _p(words), _p(g64), _p(self.s), ctypes.c_float(self.mean_s), self.n, _p(F), self.dg.sp())
        return F


class ProposalNet:
    """The network's parameters (float32 master + bf16 copy) and its forward,
    backward and Adam step, all through libpqi kernels."""

    def __init__(self, device=None, seed: int = 0, params: np.ndarray | None = None):
        self.device = torch.device(device) if device is not None else D.default_device()
        self.layout, self.count = param_layout()
        if params is None:
            from_oracle_style = _init_params(seed)
            params = from_oracle_style
        self.w = torch.from_numpy(np.asarray(params, dtype=np.float32)).to(self.device)
        self.w16 = torch.empty(self.count, dtype=torch.bfloat16, device=self.device)
        _lib.call("pqi_mpnn_to_bf16", _p(self.w), self.count, _p(self.w16), None)
        self.g = torch.zeros(self.count, dtype=torch.float32, device=self.device)
        self.m = torch.zeros(self.count, dtype=torch.float32, device=self.device)
        self.v = torch.zeros(self.count, dtype=torch.float32, device=self.device)
        self.step_count = 0

    # views ------------------------------------------------------------------------
    def _off(self, name):
        return self.layout[name][0]

    def w16_ptr(self, name):
        return ctypes.c_void_p(self.w16.data_ptr() + 2 * self._off(name))

    def w32_ptr(self, name):
        return ctypes.c_void_p(self.w.data_ptr() + 4 * self._off(name))

    def g32_ptr(self, name):
        return ctypes.c_void_p(self.g.data_ptr() + 4 * self._off(name))

    # forward / backward -----------------------------------------------------------
    tensor_cores = True  # message products on tcgen05 (False: the CUDA-core GEMM)

    def _adj(self, ctx: "GraphContext", X, ldx, beta, out32, out16, ldo, sp, what):
        """OUT[:, 0:64] = A_hat X (+ beta OUT32): the message product, on the
        tensor cores (X transposed first) or on the CUDA-core GEMM."""
        lib = _lib.load()
        Xp = X if isinstance(X, ctypes.c_void_p) else _p(X)
        if self.tensor_cores:
            Xt = torch.empty(HID * ctx.ld, dtype=torch.bfloat16, device=self.device)
            rc = lib.pqi_mpnn_transpose64(Xp, ctx.n, ldx, _p(Xt), ctx.ld, sp)
            if rc == 0:
                rc = lib.pqi_mpnn_adj_gemm(_p(ctx.Ah), ctx.ld, ctx.n, _p(Xt), ctx.ld, ctypes.c_float(beta),
                                           out32 if out32 is not None else None, out16, ldo, sp)
        else:
            rc = lib.pqi_mpnn_gemm(0, 0, ctx.n, HID, ctx.n, ctypes.c_float(1.0), _p(ctx.Ah), ctx.ld, Xp, ldx,
                                   ctypes.c_float(beta), out32, out16, ldo, None, 0, sp)
        if rc:
            raise _lib.PQIError(rc, what)

    def forward(self, ctx: GraphContext, F: torch.Tensor, stream=None):
        """Logits (float32, n) and the activations the backward pass needs."""
        n = ctx.n
        dev = self.device
        sp = D.stream_ptr(stream)
        gemm = _lib.load().pqi_mpnn_gemm
        C = [torch.empty(n * 2 * HID, dtype=torch.bfloat16, device=dev) for _ in range(LAYERS + 1)]
        H32 = [torch.empty(n * 2 * HID, dtype=torch.float32, device=dev) for _ in range(LAYERS + 1)]
        ld2 = 2 * HID

        def chk(rc, what):
            if rc:
                raise _lib.PQIError(rc, what)

        # H0 = relu(F A0 + b0) -> left half of C[0]
        chk(gemm(0, 0, n, HID, FEAT, 1.0, _p(F), FEAT, self.w16_ptr("A0"), HID, 0.0, _p(H32[0]), _p(C[0]), ld2, self.w32_ptr("b0"), 1, sp), "gemm A0")
        for l in range(1, LAYERS + 1):
            Cl = C[l - 1]
            # M = A_hat H_{l-1} -> right half of C[l-1]
            self._adj(ctx, Cl, ld2, 0.0, None, ctypes.c_void_p(Cl.data_ptr() + 2 * HID), ld2, sp, f"msg{l}")
            # H_l = relu(C AB_l + b_l) -> left half of C[l]
            chk(gemm(0, 0, n, HID, 2 * HID, 1.0, _p(Cl), ld2, self.w16_ptr(f"AB{l}"), HID, 0.0, _p(H32[l]), _p(C[l]), ld2, self.w32_ptr(f"b{l}"), 1, sp), f"gemm AB{l}")
        logits = torch.empty(n, dtype=torch.float32, device=dev)
        chk(gemm(0, 0, n, 1, HID, 1.0, _p(C[LAYERS]), ld2, self.w16_ptr("c"), 1, 0.0, _p(logits), None, 1, self.w32_ptr("c0"), 0, sp), "gemm out")
        return logits, {"F": F, "C": C, "H32": H32}

    def backward(self, ctx: GraphContext, cache, dlogits: torch.Tensor, stream=None):
        """Accumulate the parameter gradients of one graph into self.g."""
        n = ctx.n
        dev = self.device
        sp = D.stream_ptr(stream)
        lib = _lib.load()
        gemm = lib.pqi_mpnn_gemm
        ld2 = 2 * HID
        C, H32 = cache["C"], cache["H32"]

        def chk(rc, what):
            if rc:
                raise _lib.PQIError(rc, what)

        dl16 = torch.empty(n, dtype=torch.bfloat16, device=dev)
        chk(lib.pqi_mpnn_to_bf16(_p(dlogits), n, _p(dl16), sp), "dl16")
        # dc += H3^T dl ; dc0 += sum dl
        chk(gemm(1, 0, HID, 1, n, 1.0, _p(C[LAYERS]), ld2, _p(dl16), 1, 1.0, self.g32_ptr("c"), None, 1, None, 0, sp), "dc")
        chk(lib.pqi_mpnn_colsum(_p(dlogits), n, 1, 1, self.g32_ptr("c0"), 1, sp), "dc0")
        # dH3 = dl c^T
        dH = torch.empty(n * ld2, dtype=torch.float32, device=dev)
        chk(gemm(0, 0, n, HID, 1, 1.0, _p(dl16), 1, self.w16_ptr("c"), HID, 0.0, _p(dH), None, ld2, None, 0, sp), "dH3")
        dZ = torch.empty(n * ld2, dtype=torch.float32, device=dev)
        dZ16 = torch.empty(n * ld2, dtype=torch.bfloat16, device=dev)
        dC = torch.empty(n * ld2, dtype=torch.float32, device=dev)
        dC16 = torch.empty(n * ld2, dtype=torch.bfloat16, device=dev)
        for l in range(LAYERS, 0, -1):
            chk(lib.pqi_mpnn_relu_bwd(_p(dH), _p(H32[l]), n * ld2, _p(dZ), _p(dZ16), sp), "relu")
            Cl = C[l - 1]
            # dAB_l += C^T dZ ; db_l += colsum dZ
            chk(gemm(1, 0, 2 * HID, HID, n, 1.0, _p(Cl), ld2, _p(dZ16), ld2, 1.0, self.g32_ptr(f"AB{l}"), None, HID, None, 0, sp), f"dAB{l}")
            chk(lib.pqi_mpnn_colsum(_p(dZ), n, HID, ld2, self.g32_ptr(f"b{l}"), 1, sp), f"db{l}")
            # dC = dZ AB_l^T
            chk(gemm(0, 1, n, 2 * HID, HID, 1.0, _p(dZ16), ld2, self.w16_ptr(f"AB{l}"), HID, 0.0, _p(dC), _p(dC16), ld2, None, 0, sp), f"dC{l}")
            # dH_{l-1} = dC[:, :64] + A_hat dC[:, 64:]   (A_hat symmetric)
            self._adj(ctx, ctypes.c_void_p(dC16.data_ptr() + 2 * HID), ld2, 1.0, _p(dC), None, ld2, sp, f"dmsg{l}")
            dH, dC = dC, dH
        chk(lib.pqi_mpnn_relu_bwd(_p(dH), _p(H32[0]), n * ld2, _p(dZ), _p(dZ16), sp), "relu0")
        chk(gemm(1, 0, FEAT, HID, n, 1.0, _p(cache["F"]), FEAT, _p(dZ16), ld2, 1.0, self.g32_ptr("A0"), None, HID, None, 0, sp), "dA0")
        chk(lib.pqi_mpnn_colsum(_p(dZ), n, HID, ld2, self.g32_ptr("b0"), 1, sp), "db0")

    def loss_grad(self, logits: torch.Tensor, target: torch.Tensor | None, stream=None):
        n = logits.numel()
        if target is not None:
            target = target.to(device=self.device, dtype=torch.float32).contiguous()
            if target.numel() != n:
                raise ValueError("target and logits differ in length")
        loss = torch.empty(1, dtype=torch.float32, device=self.device)
        dl = torch.empty(n, dtype=torch.float32, device=self.device)
        prob = torch.empty(n, dtype=torch.float32, device=self.device)
        _lib.call("pqi_mpnn_softmax_xent", _p(logits), _p(target), n, _p(loss), _p(dl), _p(prob), D.stream_ptr(stream))
        return loss, dl, prob

    def zero_grad(self):
        self.g.zero_()

    def clip_grad(self, max_norm: float) -> float:
        """Scale the gradient to at most `max_norm` (L2); returns the norm before."""
        norm = torch.empty(1, dtype=torch.float32, device=self.device)
        _lib.call("pqi_mpnn_grad_clip", _p(self.g), self.count, ctypes.c_float(max(0.0, float(max_norm))), _p(norm),
                  None)
        return float(norm.item())

    def adam_step(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, stream=None):
        self.step_count += 1
        _lib.call("pqi_mpnn_adam", _p(self.w), _p(self.g), _p(self.m), _p(self.v), _p(self.w16), self.count,
                  ctypes.c_float(lr), ctypes.c_float(b1), ctypes.c_float(b2), ctypes.c_float(eps), self.step_count, D.stream_ptr(stream))

    # inference --------------------------------------------------------------------
    def proposal(self, ctx: GraphContext, words: torch.Tensor, g64=None):
        """Softmax proposal (float32, n) for the state `words`."""
        F = ctx.features(words, g64)
        logits, _ = self.forward(ctx, F)
        _, _, prob = self.loss_grad(logits, None)
        return prob

    def snapshot(self):
        """Copy of the parameters (float32 master)."""
        return self.w.detach().clone()

    def restore(self, params: torch.Tensor, reset_moments: bool = True):
        """Load parameters from `snapshot()`, refresh the bf16 copy and, by
        default, reset Adam's moments."""
        self.w.copy_(params)
        _lib.call("pqi_mpnn_to_bf16", _p(self.w), self.count, _p(self.w16), None)
        if reset_moments:
            self.m.zero_()
            self.v.zero_()

    def state_dict(self):
        return {"params": self.w.detach().cpu().clone(), "step": self.step_count}

    def save(self, path):
        torch.save(self.state_dict(), path)

    @classmethod
    def load(cls, path, device=None):
        sd = torch.load(path, map_location="cpu")
        net = cls(device=device, params=sd["params"].numpy())
        net.step_count = int(sd.get("step", 0))
        return net


def _init_params(seed=0):
    lay, total = param_layout()
    rng = np.random.default_rng(seed)
    th = np.zeros(total)
    for name, (o, s) in lay.items():
        size = int(np.prod(s))
        if name.startswith("A"):
            th[o : o + size] = rng.standard_normal(size) * np.sqrt(2.0 / s[0])
        elif name == "c":
            th[o : o + size] = rng.standard_normal(size) * np.sqrt(1.0 / HID)
        else:
            th[o : o + size] = 0.01
    return th


def task_proposals(net: "ProposalNet", dg: D.DeviceGraph, words: torch.Tensor, temperature: float = 3.0,
                   mix: float = 0.0):
    """One kick distribution per task, from each task's own state: returns
    (concatenated normalised cumulative arrays, float64; per-task offsets,
    int64). The proposal softmax(logit) flattened by the temperature
    (softmax(logit / T), i.e. p^(1/T) renormalised) and mixed with the uniform
    distribution (weight `mix`), built on the device by pqi_mpnn_kick_cdf; a
    non-finite output becomes uniform, so the search never depends on the
    network being right."""
    ctx = GraphContext(dg)
    n = dg.n
    tasks = int(words.shape[0])
    logits = torch.empty(tasks * n, dtype=torch.float32, device=words.device)
    for t in range(tasks):
        F = ctx.features(words[t].contiguous())
        lg, _ = net.forward(ctx, F)
        logits[t * n:(t + 1) * n].copy_(lg)
    cdf = torch.empty(tasks * n, dtype=torch.float64, device=words.device)
    _lib.call("pqi_mpnn_kick_cdf", _p(logits), n, tasks, ctypes.c_float(temperature), ctypes.c_float(mix), _p(cdf),
              dg.sp())
    off = torch.arange(tasks, dtype=torch.int64, device=words.device) * n
    return cdf, off


# ------------------------------------------------------------------------------------
# Training data from the search itself, and training


def make_examples(dgs, tasks_per_graph=4, rounds=12, kick_frac=1 / 16, seed=0):
    """(graph index, local optimum A as device words, target distribution) for
    each task whose iterated search found a better optimum B: target = uniform
    over the nodes where A and B differ."""
    from .batch import BatchedSearch

    out = []
    by_kind = {}
    for i, dg in enumerate(dgs):
        by_kind.setdefault(dg.w.kind, []).append(i)
    for kind, idx in by_kind.items():
        group = [dgs[i] for i in idx]
        bs = BatchedSearch(group)
        tg = [g for g in range(len(group)) for _ in range(tasks_per_graph)]
        words0 = bs.random_states(tg, seed=seed + 17 * kind)
        spin = 1
        vA, wA, _, _ = bs.run(tg, words0, spin, rounds=0)
        kick = max(2, int(round(min(g.n for g in group) * kick_frac)))
        vB, wB, _, _ = bs.run(tg, wA.reshape(-1).contiguous(), spin, rounds=rounds, kick=kick, seed=seed + 1)
        better = (vB > vA + 1e-9).cpu().numpy()
        A = bs.unpack(wA, tg)
        B = bs.unpack(wB, tg)
        for t, g in enumerate(tg):
            if not better[t]:
                continue
            diff = A[t] != B[t]
            if not diff.any():
                continue
            tgt = (diff / diff.sum()).astype(np.float32)
            out.append((idx[g], A[t], tgt))
    return out


def train(net: ProposalNet, dgs, examples, epochs=2, lr=2e-3, batch=8, log=None, clip=1.0):
    """Adam on the softmax cross-entropy of the examples; returns loss history.
    `lr` is a number or a function of the optimiser step; gradients are
    clipped to L2 norm `clip` (0: off)."""
    ctxs = {}
    hist = []
    order = np.arange(len(examples))
    rng = np.random.default_rng(0)
    for ep in range(epochs):
        rng.shuffle(order)
        for b0 in range(0, len(order), batch):
            net.zero_grad()
            tot = 0.0
            losses = []
            for j in order[b0 : b0 + batch]:
                gi, bits, tgt = examples[j]
                dg = dgs[gi]
                if gi not in ctxs:
                    ctxs[gi] = GraphContext(dg)
                ctx = ctxs[gi]
                words = dg.pack(bits)
                F = ctx.features(words)
                logits, cache = net.forward(ctx, F)
                t = torch.from_numpy(tgt).to(net.device)
                loss, dl, _ = net.loss_grad(logits, t)
                dl /= len(order[b0 : b0 + batch])
                net.backward(ctx, cache, dl)
                losses.append(loss)
            if clip:
                net.clip_grad(clip)
            net.adam_step(lr=lr(net.step_count) if callable(lr) else lr)
            tot = float(torch.stack(losses).mean().item())
            hist.append(tot)
            if log is not None and (len(hist) % 50 == 0):
                log(f"step {len(hist)} loss {tot:.4f}")
        if len(ctxs) > 64:
            ctxs.clear()
    return hist
