"""One proposal-network forward and backward on G(n, 0.01) N(0,1) for
profiling (ncu) the tensor-core message products; default n = 16384."""

import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import numpy as np  # noqa: E402
import torch  # noqa: E402

from pyqrackising_b200 import learned as L  # noqa: E402
from pyqrackising_b200 import workloads as wl  # noqa: E402
from pyqrackising_b200.device import DeviceGraph  # noqa: E402

n = int(sys.argv[1]) if len(sys.argv) > 1 else 16384
dg = DeviceGraph(wl.gnp_weighted(n, 0.01, seed=5, dist="normal"))
ctx = L.GraphContext(dg)
net = L.ProposalNet(seed=1)
F = ctx.features(dg.pack(np.random.default_rng(1).random(n) < 0.5))
logits, cache = net.forward(ctx, F)
_, dl, _ = net.loss_grad(logits, torch.full((n,), 1.0 / n, device="cuda"))
net.backward(ctx, cache, dl)
torch.cuda.synchronize()
ok = bool(torch.isfinite(logits).all().item()) and bool(torch.isfinite(net.g).all().item())
print({"n": n, "finite": ok})
sys.exit(0 if ok else 1)
