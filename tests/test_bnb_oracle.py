"""The branch-and-bound oracle (oracle/bnb_oracle.py) against the reference's
own results (tests/golden/golden_bnb.npz, made by
tests/golden/make_bnb_golden.py) and against exhaustive search."""

import itertools
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden", "golden_bnb.npz")


def _cases():
    z = np.load(GOLD)
    return z, [str(s) for s in z["names"]]


def test_oracle_reproduces_the_reference_results():
    from oracle import bnb_oracle as B

    z, names = _cases()
    cap = int(z["batch_cap"])
    for name in names:
        W = z[f"{name}_W"]
        spin = bool(z[f"{name}_spin"])
        bits, cut, energy, certified = B.solve(W, str(z[f"{name}_guess"]), spin, cap)
        assert bits == str(z[f"{name}_bits"]), name
        assert cut == pytest.approx(float(z[f"{name}_cut"]), rel=1e-6, abs=1e-6), name
        assert energy == pytest.approx(float(z[f"{name}_energy"]), rel=1e-6, abs=1e-6), name
        assert certified == bool(z[f"{name}_certified"])


def test_oracle_maxcut_value_is_the_exhaustive_optimum():
    from oracle import bnb_oracle as B

    z, names = _cases()
    for name in names:
        W = z[f"{name}_W"]
        if bool(z[f"{name}_spin"]) or W.shape[0] > 14:
            continue
        n = W.shape[0]
        best = max(B.objectives(W, np.array(bits, dtype=bool))[0]
                   for bits in itertools.product([0, 1], repeat=n))
        _, cut, _, _ = B.solve(W, str(z[f"{name}_guess"]), False, int(z["batch_cap"]))
        assert cut == pytest.approx(best, rel=1e-6, abs=1e-6), name
