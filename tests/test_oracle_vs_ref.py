"""The C restatement against the reference's kernels.cl compiled for the host
(oracle/_ref) on fresh random instances, including ragged n, non-power-of-two
local sizes and ties. Skipped when oracle/_ref was not built."""

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (needs the reference source)")


def _sym(rng, n, kind):
    if kind == "pm1":
        A = rng.choice([-1.0, 0.0, 1.0], size=(n, n), p=[0.2, 0.6, 0.2])
    elif kind == "unit":
        A = (rng.random((n, n)) < 0.5).astype(np.float64)
    else:
        A = rng.standard_normal((n, n))
    A = np.triu(A, 1)
    return (A + A.T).astype(np.float32)


@pytest.mark.parametrize("n", [24, 27, 31, 40, 64, 100, 129])
@pytest.mark.parametrize("kind", ["pm1", "unit", "normal"])
def test_flips_cut_gray(n, kind):
    rng = np.random.default_rng(n * 7 + len(kind))
    W = _sym(rng, n, kind)
    th = rng.random(n) < 0.5
    th32 = O.pack32(th)
    for spin in (0, 1):
        for mpe in (148, 7, 40):
            G, L = O.flip_geometry(n, mpe)
            a = O.single_select(W, th32, spin, G, L)
            b = O.ref_single_select(W, th32, spin, G, L)
            assert (a[0], a[1]) == (b[0], b[1])
            a = O.double_select(W, th32, spin, G, L)
            b = O.ref_double_select(W, th32, spin, G, L)
            assert (a[0], a[1]) == (b[0], b[1])
        X = rng.random((96, n)) < 0.5
        G, L = O.cut_geometry(96, 148)
        a = O.cut_select(W, O.pack32(X), 96, spin, G, L)
        b = O.ref_cut_select(W, O.pack32(X), 96, spin, G, L)
        assert (a[0], a[1]) == (b[0], b[1])
        for G, T in ((148, 40), (37, 5), (300, 301)):
            if O.gray_has_oob(n, T, G):
                continue
            t1, e1, _ = O.gray(W, O.pack64(th), spin, T, G)
            t2, e2 = O.ref_gray(W, O.pack64(th), spin, T, G)
            assert np.array_equal(t1, t2)
            assert np.array_equal(e1.view(np.uint32), e2.view(np.uint32))
