"""Small cluster-ascent run for profiling (ncu): SK n=8192, 8 starts, 8-CTA
clusters; exits non-zero if the result disagrees with the batched kernel."""

import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import torch  # noqa: E402

from pyqrackising_b200 import workloads as wl  # noqa: E402
from pyqrackising_b200.batch import BatchedSearch  # noqa: E402
from pyqrackising_b200.device import DeviceGraph  # noqa: E402

n = int(sys.argv[1]) if len(sys.argv) > 1 else 8192
starts = int(sys.argv[2]) if len(sys.argv) > 2 else 8
bs = BatchedSearch([DeviceGraph(wl.sherrington_kirkpatrick(n, seed=1))])
tasks = [0] * starts
w0 = bs.random_states(tasks, seed=7)
v, best, flips, st = bs.cluster_ascent(tasks, w0, True, cluster_size=8)
v2, best2, flips2, st2 = bs.run(tasks, w0, True, rounds=0)
torch.cuda.synchronize()
ok = torch.equal(best, best2) and int(st.item()) == 0
print({"flips": int(flips.item()), "best": float(v.max()), "matches_batched": ok})
sys.exit(0 if ok else 1)
