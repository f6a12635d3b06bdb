import glob
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (runs through libpqi on cuda:0)")


def golden_names():
    return sorted(os.path.basename(p)[len("golden_"):-4] for p in glob.glob(os.path.join(GOLDEN, "golden_c*.npz")))


def load_golden(name):
    with np.load(os.path.join(GOLDEN, f"golden_{name}.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O

    O.build_oracle()
    return O
