"""The oracle's restatement of the reference's CPU candidate scoring (the CPU
baseline's workload) against values the reference itself produced."""

import numpy as np
import pytest

from conftest import GOLDEN

numba_port = pytest.importorskip("oracle.numba_port")


@pytest.mark.parametrize("name", ["er300", "sk200", "gnp257"])
def test_cut_change_matches_reference(name):
    if not numba_port.available():
        pytest.skip("numba is not installed")
    with np.load(f"{GOLDEN}/golden_numba_cutdiff.npz") as z:
        W, base, cand = z[f"{name}_W"], z[f"{name}_base"], z[f"{name}_cand"]
        vals, cuts = z[f"{name}_values"], z[f"{name}_cuts"]
    for i in range(len(base)):
        assert numba_port.cut_change(base[i], cand[i], W) == vals[i]
    assert np.array_equal(numba_port.score_batch(cand, W), cuts)
    got = numba_port.score_batch(cand, W, base=base[0])
    assert got[0] == vals[0]
    assert numba_port.select_first_max(cuts) == (float(cuts.max()), int(np.argmax(cuts)))
