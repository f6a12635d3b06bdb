"""TEST INFRASTRUCTURE ONLY: float64 CPU oracle of the learned flip-proposal
network (forward, backward, finite-difference check).

The network has no reference counterpart; this oracle restates the model the
GPU kernels implement (pyqrackising_b200/learned.py) in numpy float64 so the
kernels' gradients can be checked. Parameter layout (one flat vector):

    A0 (4 x 64), b0 (64), then for l = 1..3: AB_l (128 x 64), b_l (64),
    then c (64), c0 (1)

    A_hat = D^-1/2 W D^-1/2 (zero diagonal), D = diag(sum_{u != v} |W_vu|)
    H0 = relu(F A0 + b0)
    H_l = relu([H_{l-1}, A_hat H_{l-1}] AB_l + b_l),  l = 1..3
    logits = H_3 c + c0
    loss = -sum_v t_v log softmax(logits)_v
"""

from __future__ import annotations

import numpy as np

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


def unpack(theta):
    lay, _ = param_layout()
    return {k: theta[o : o + int(np.prod(s))].reshape(s) for k, (o, s) in lay.items()}


def norm_adj(W):
    W = np.asarray(W, dtype=np.float64).copy()
    np.fill_diagonal(W, 0.0)
    s = np.abs(W).sum(axis=1)
    d = np.sqrt(np.maximum(s, 1e-30))
    return W / d[:, None] / d[None, :], s


def features(bits, W, s):
    Wd = np.asarray(W, dtype=np.float64).copy()
    np.fill_diagonal(Wd, 0.0)
    x = np.where(bits, 1.0, -1.0)
    g = x * (Wd @ x)
    sv = np.maximum(s, 1e-30)
    return np.stack([x, g / sv, sv / max(s.mean(), 1e-30), np.ones_like(x)], axis=1)


def _ident(x):
    return x


def bf16_round(x):
    """Round float64 values to bfloat16 (round to nearest even), as the GPU
    kernels do where they store bf16 (used to mirror their precision)."""
    a = np.asarray(x, dtype=np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(theta, F, Ah, q=_ident):
    """q rounds the values the GPU stores in bf16 (identity = pure float64)."""
    p = unpack(theta)
    cache = {"F": F}
    Z = F @ p["A0"] + p["b0"]
    H = np.maximum(Z, 0.0)
    cache["H0"] = H
    Hq = q(H)
    for l in range(1, LAYERS + 1):
        C = np.concatenate([Hq, q(Ah @ Hq)], axis=1)
        Z = C @ p[f"AB{l}"] + p[f"b{l}"]
        H = np.maximum(Z, 0.0)
        Hq = q(H)
        cache[f"C{l}"] = C
        cache[f"H{l}"] = H
    cache["Hq_last"] = Hq
    logits = Hq @ p["c"] + p["c0"][0]
    return logits, cache


def loss_and_dlogits(logits, t):
    z = logits - logits.max()
    lse = np.log(np.exp(z).sum())
    logp = z - lse
    return float(-(t * logp).sum()), np.exp(logp) - t


def backward(theta, cache, Ah, dlogits, q=_ident):
    p = unpack(theta)
    lay, total = param_layout()
    g = np.zeros(total)

    def put(name, val):
        o, s = lay[name]
        g[o : o + int(np.prod(s))] = val.reshape(-1)

    H = cache["Hq_last"]
    dlq = q(dlogits)
    put("c", H.T @ dlq)
    put("c0", np.array([dlogits.sum()]))
    dH = np.outer(dlq, p["c"])
    for l in range(LAYERS, 0, -1):
        dZ = dH * (cache[f"H{l}"] > 0)
        dZq = q(dZ)
        C = cache[f"C{l}"]
        put(f"AB{l}", C.T @ dZq)
        put(f"b{l}", dZ.sum(axis=0))
        dC = dZq @ p[f"AB{l}"].T
        dH = dC[:, :HID] + Ah.T @ q(dC[:, HID:])
    dZ = dH * (cache["H0"] > 0)
    put("A0", cache["F"].T @ q(dZ))
    put("b0", dZ.sum(axis=0))
    return g


def loss_fn(theta, F, Ah, t):
    logits, _ = forward(theta, F, Ah)
    return loss_and_dlogits(logits, t)[0]


def init_params(seed=0):
    lay, total = param_layout()
    rng = np.random.default_rng(seed)
    th = np.zeros(total)
    for name, (o, s) in lay.items():
        if name.startswith("A"):
            fan_in = s[0]
            th[o : o + int(np.prod(s))] = rng.standard_normal(int(np.prod(s))) * np.sqrt(2.0 / fan_in)
        elif name == "c":
            th[o : o + int(np.prod(s))] = rng.standard_normal(int(np.prod(s))) * np.sqrt(1.0 / HID)
        else:
            th[o : o + int(np.prod(s))] = 0.01
    return th


def finite_difference_check(theta, F, Ah, t, idx, eps=1e-6):
    """Central differences of the loss at parameter indices idx; returns
    (numeric, analytic) arrays."""
    logits, cache = forward(theta, F, Ah)
    _, dl = loss_and_dlogits(logits, t)
    ana = backward(theta, cache, Ah, dl)[idx]
    num = np.empty(len(idx))
    for j, i in enumerate(idx):
        tp = theta.copy()
        tp[i] += eps
        tm = theta.copy()
        tm[i] -= eps
        num[j] = (loss_fn(tp, F, Ah, t) - loss_fn(tm, F, Ah, t)) / (2 * eps)
    return num, ana
