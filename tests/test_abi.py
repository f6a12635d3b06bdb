"""The C ABI library loads and exports every entry point include/pqi.h declares,
and its host-side selection reproduces the reference's reduction (no GPU)."""

import ctypes
import os
import re

import numpy as np
import pytest

from conftest import REPO


def header_functions():
    src = open(os.path.join(REPO, "include", "pqi.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pqi_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from pyqrackising_b200 import _lib

    lib = _lib.load()
    names = header_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(_lib.SIGNATURES), "ctypes signatures out of sync with include/pqi.h"


def test_host_queries():
    from pyqrackising_b200 import _lib

    lib = _lib.load()
    assert lib.pqi_version().startswith(b"libpqi")
    assert lib.pqi_padded_ld(1) == 128 and lib.pqi_padded_ld(129) == 256
    assert lib.pqi_workspace_bytes(2048, 4096) > 4096 * 2048


def _host_select(values, G, L):
    from pyqrackising_b200 import _lib

    v = np.ascontiguousarray(values, dtype=np.float32)
    e = ctypes.c_float()
    i = ctypes.c_int()
    rc = _lib.load().pqi_select_host(v.ctypes.data, v.size, G, L, ctypes.byref(e), ctypes.byref(i))
    return rc, e.value, i.value


@pytest.mark.parametrize("count", [1, 5, 24, 31, 32, 100, 1000, 4097])
@pytest.mark.parametrize("G,L", [(160, 32), (32, 32), (24, 24), (30, 30), (20, 20), (7, 1), (148, 1), (96, 32)])
def test_selection_key_matches_reference_tree(oracle_mod, count, G, L):
    """Ties everywhere (integer values drawn from a tiny range) so the tie rule decides."""
    rng = np.random.default_rng(count * 31 + G + L)
    for trial in range(5):
        vals = rng.integers(-2, 3, size=count).astype(np.float32)
        if trial == 4:
            vals[:] = 1.0
        rc, e, i = _host_select(vals, G, L)
        assert rc == 0
        oe, oi = oracle_mod.select(vals, G, L)
        if oi >= count:  # all candidates dropped by a non power-of-two tree: the slot id is reported
            continue
        assert (np.float32(e), i) == (oe, oi), (vals.tolist(), G, L)


def test_selection_rejects_bad_geometry():
    rc, _, _ = _host_select(np.zeros(8, np.float32), 10, 3)
    assert rc == 1
    rc, _, _ = _host_select(np.zeros(8, np.float32), 256, 128)
    assert rc == 1


def test_no_cpu_fallback_without_library(monkeypatch, tmp_path):
    from pyqrackising_b200 import _lib

    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(_lib.PQIUnavailable):
        _lib.load(str(tmp_path / "missing.so"))


def test_graph_descriptor_layout_matches_the_library():
    """The batched entry points read an array of C structs; the host packs it
    with a numpy dtype. Size and field offsets must agree (the row-list
    pointers follow upper_sum)."""
    from pyqrackising_b200 import _lib
    from pyqrackising_b200.batch import _DESC

    assert _lib.load().pqi_batch_graph_desc_bytes() == _DESC.itemsize == 56
    offsets = {name: _DESC.fields[name][1] for name in _DESC.names}
    assert offsets == {"W": 0, "n": 8, "ld": 12, "kind": 16, "pad": 20, "upper_sum": 24,
                       "adj_ptr": 32, "adj_col": 40, "adj_val": 48}
