"""Tile-major item order, host side: the tables a launch of several jobs
uses (gexs_debug_tile_order returns the ones the launch path builds) and a
Python restatement of the device decode (tile_job in
gexs_b200/csrc/gexs_tiles.cuh).  Every flat item must map to one (job,
tile) with tile < that job's tile count, every such pair must be hit once,
and the items must run row by row (tile 0 of every job that has one, then
tile 1, ...).  Tile counts are uneven, with zeros, ties and one job."""
import ctypes as C

import numpy as np
import pytest

from gexs_b200 import _capi as capi


def _tables(tiles):
    nj = len(tiles)
    t = (C.c_int32 * nj)(*tiles)
    out = (C.c_int32 * (3 * nj + 1))()
    assert capi.lib().gexs_debug_tile_order(t, nj, out) == capi.GEXS_OK
    o = np.frombuffer(out, dtype=np.int32).astype(np.int64)
    return o[:nj + 1], o[nj + 1:2 * nj + 1], o[2 * nj + 1:]


def _decode(F, R, P, ti):
    """tile_job's tile-major branch: last segment whose start is <= ti,
    then the row and the rank within it"""
    nj = len(P)
    lo, hi = 0, nj
    while hi - lo > 1:
        m = (lo + hi) >> 1
        if F[m] <= ti:
            lo = m
        else:
            hi = m
    act = nj - lo
    d = ti - F[lo]
    return int(P[d % act]), int(R[lo] + d // act)


CASES = [
    [5],
    [3, 3, 3],
    [7, 1, 4, 4, 0, 9, 2],
    [0, 0, 6],
    [1] * 64,
]


@pytest.mark.parametrize("tiles", CASES + [list(np.random.default_rng(s).integers(0, 40, size=n))
                                           for s, n in ((1, 5), (2, 17), (3, 64))])
def test_tile_major_tables_are_a_row_major_bijection(tiles):
    tiles = [int(v) for v in tiles]
    F, R, P = _tables(tiles)
    total = sum(tiles)
    assert F[0] == 0 and F[-1] == total
    assert sorted(P.tolist()) == list(range(len(tiles)))
    seen = [_decode(F, R, P, i) for i in range(total)]
    assert len(set(seen)) == total
    assert all(0 <= t < tiles[j] for j, t in seen)
    rows = [t for _, t in seen]
    assert rows == sorted(rows)                        # row by row
    for r in set(rows):                                # every job with a tile r is in row r
        assert sorted(j for j, t in seen if t == r) == sorted(j for j, n in enumerate(tiles) if n > r)


def test_tile_order_rejects_bad_arguments():
    out = (C.c_int32 * 4)()
    t = (C.c_int32 * 1)(-1)
    assert capi.lib().gexs_debug_tile_order(t, 1, out) == capi.GEXS_ERR_INVALID
    assert capi.lib().gexs_debug_tile_order(t, 0, out) == capi.GEXS_ERR_INVALID
