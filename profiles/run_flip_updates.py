"""Batched-ascent run for profiling (ncu): SK n=8192 float32; arguments:
starts (default 444, one resident wave at 3 per SM), flip budget per start
(default 64), local-field precision f64 | f32 (default f64). Exits non-zero on
a bad status."""

import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import numpy as np  # noqa: E402
import torch  # noqa: E402

from pyqrackising_b200 import workloads as wl  # noqa: E402
from pyqrackising_b200.batch import BatchedSearch  # noqa: E402
from pyqrackising_b200.device import DeviceGraph  # noqa: E402

tasks = int(sys.argv[1]) if len(sys.argv) > 1 else 444
budget = int(sys.argv[2]) if len(sys.argv) > 2 else 64
fields = sys.argv[3] if len(sys.argv) > 3 else "f64"
bs = BatchedSearch([DeviceGraph(wl.sherrington_kirkpatrick(8192, seed=1))])
tg = torch.zeros(tasks, dtype=torch.int32, device="cuda")
w0 = bs.random_states(np.zeros(tasks, dtype=np.int32), seed=5)
for _ in range(2):
    v, _, flips, st = bs.run(tg, w0, True, rounds=0, flip_budget=budget, fields=fields)
torch.cuda.synchronize()
print({"flips": int(flips.item()), "status": int(st.item())})
sys.exit(0 if int(st.item()) in (0, 3) else 1)  # 3: the flip budget ran out, as intended
