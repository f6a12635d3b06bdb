"""The double pass's tile runs (pyqrackising_b200/csrc/pqi_core.cu, TileWalk),
restated on the host: the kept tiles of the upper triangle (row groups of DR
rows x column chunks of CW columns, a tile kept when it reaches above the
diagonal) are cut into one contiguous run per CTA in row-group-major order; a
run's start comes from the closed-form count of kept tiles before a row group
and a binary search. Every kept tile must be walked exactly once, by any grid,
for every n the pass accepts (2 .. 46341), both tile shapes (float32: 16 rows x
1024 columns; int8: 8 rows x 4096 columns)."""

import numpy as np
import pytest


def kept_tiles(n, cw, dr):
    ng, nc = (n - 1 + dr - 1) // dr, (n + cw - 1) // cw
    return [(rg, c) for rg in range(ng) for c in range(nc) if (c + 1) * cw > rg * dr + 1]


def runs(n, cw, dr, grid):
    ng, nc, q = (n - 1 + dr - 1) // dr, (n + cw - 1) // cw, cw // dr

    def prefix(r):  # kept tiles of row groups 0 .. r-1 (row group g keeps chunks g // q .. nc-1)
        a, b = r // q, r % q
        return r * nc - (q * a * (a - 1) // 2 + a * b)

    total = prefix(ng)
    per = (total + grid - 1) // grid
    out = []
    for blk in range(grid):
        t0 = blk * per
        left = max(0, min(total, t0 + per) - t0)
        if not left:
            continue
        lo, hi = 0, ng - 1
        while lo < hi:
            mid = (lo + hi + 1) >> 1
            if prefix(mid) <= t0:
                lo = mid
            else:
                hi = mid - 1
        rg, c = lo, lo // q + (t0 - prefix(lo))
        while left:
            out.append((blk, rg, c))
            left -= 1
            c += 1
            if c == nc:
                rg += 1
                c = rg // q
    return out


@pytest.mark.parametrize("shape", [(1024, 16), (4096, 8)])
@pytest.mark.parametrize("n", [2, 3, 17, 100, 1023, 1024, 1025, 2048, 4097, 8192, 12345])
def test_runs_cover_every_kept_tile_once(n, shape):
    cw, dr = shape
    want = kept_tiles(n, cw, dr)
    for grid in (1, 7, 148, 296):
        got = runs(n, cw, dr, grid)
        tiles = [(rg, c) for _, rg, c in got]
        assert sorted(tiles) == sorted(want) and len(tiles) == len(set(tiles))
        # each CTA's run is contiguous in row-group-major order
        order = {t: i for i, t in enumerate(sorted(want))}
        for blk in {b for b, _, _ in got}:
            idx = [order[(rg, c)] for b, rg, c in got if b == blk]
            assert idx == list(range(idx[0], idx[0] + len(idx)))


def test_prefix_count_at_the_largest_n():
    """The closed-form count against a direct sum at n = 46341 (the pass's
    largest), where the counts reach the tens of thousands."""
    n = 46341
    for cw, dr in ((1024, 16), (4096, 8)):
        ng, nc, q = (n - 1 + dr - 1) // dr, (n + cw - 1) // cw, cw // dr
        direct = np.cumsum([0] + [nc - g // q for g in range(ng)])
        for r in (0, 1, q - 1, q, q + 1, ng // 2, ng):
            a, b = r // q, r % q
            assert r * nc - (q * a * (a - 1) // 2 + a * b) == direct[r]
        assert len(kept_tiles(n, cw, dr)) == direct[ng]
