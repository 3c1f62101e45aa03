"""Host side of the persistent tensor-core launch's work schedule (no device needed).

The launch hands work item i to CTA i % grid.  The library weighs every item by its r2 blocks (a
symmetric instance's tiles start at their diagonal block, so their items shrink with the tile index),
sorts them, the most first, and reverses every second round of grid items.  The CTAs then get about
the same number of blocks, where tiles in index order load the first CTAs most.
"""
import ctypes as C

import numpy as np
import pytest

from tcscf_b200 import ffi

BM, BK = 128, 64


def _schedule(n1, n2, sym, nsplit, grid):
    lib = ffi.lib()
    n = C.c_int()
    assert lib.tcscf_schedule_items(n1, n2, sym, nsplit, grid, None, 0, C.byref(n)) == ffi.OK
    buf = (C.c_int * (3 * n.value))()
    assert lib.tcscf_schedule_items(n1, n2, sym, nsplit, grid, buf, n.value, C.byref(n)) == ffi.OK
    return np.frombuffer(buf, dtype=np.int32).reshape(-1, 3).copy()


def _blocks(n1, n2, sym, nsplit):
    """every item's r2 blocks, restated: tile t, split s covers [jb, je) with jb = 2 t (symmetric) + s per"""
    tiles, blocks = -(-n1 // BM), -(-n2 // BK)
    per = -(-blocks // nsplit)
    out = {}
    for t in range(tiles):
        for s in range(-(-blocks // per)):
            jb = (2 * t if sym else 0) + s * per
            je = max(jb, min(jb + per, blocks))
            out[(t, s)] = je - jb
    return out


def _cta_loads(order, grid):
    loads = np.zeros(grid)
    for i, w in enumerate(order):
        loads[i % grid] += w
    return loads


@pytest.mark.parametrize("n1,sym,nsplit,grid", [(406_000, 1, 1, 148), (263_900, 1, 1, 148), (59_000, 1, 1, 148),
                                                (406_000, 0, 1, 148), (20_000, 0, 4, 148), (9_000, 1, 2, 148)])
def test_items_cover_every_tile_and_balance_the_ctas(n1, sym, nsplit, grid):
    s = _schedule(n1, n1, sym, nsplit, grid)
    ref = _blocks(n1, n1, sym, nsplit)
    # every (tile, split) exactly once, with its block count
    assert len(s) == len(ref)
    assert {(int(t), int(sp)): int(w) for t, sp, w in s} == ref
    g = min(grid, len(s))
    dealt = _cta_loads(s[:, 2], g)
    in_order = _cta_loads([ref[k] for k in sorted(ref)], g)
    assert dealt.max() <= in_order.max()
    # no CTA gets more than the mean plus one item (the bound of a list schedule; equal items still
    # leave the quantisation of items over CTAs)
    assert dealt.max() <= dealt.mean() + s[:, 2].max()


def test_kr_symmetric_schedule_figures():
    # the 406,000-point symmetric Kr build: tiles in order leave the busiest of 148 CTAs 4.7 % above
    # the mean; the dealt order 0.2 %
    s = _schedule(406_000, 406_000, 1, 1, 148)
    ref = _blocks(406_000, 406_000, 1, 1)
    dealt = _cta_loads(s[:, 2], 148)
    in_order = _cta_loads([ref[k] for k in sorted(ref)], 148)
    assert abs(in_order.max() / in_order.mean() - 1 - 0.047) < 0.002
    assert dealt.max() / dealt.mean() - 1 < 0.003


def test_schedule_argument_checks():
    lib = ffi.lib()
    n = C.c_int()
    for args in ((0, 10, 1, 1, 148), (10, 10, 1, 0, 148), (10, 10, 1, 1, 0)):
        assert lib.tcscf_schedule_items(*args, None, 0, C.byref(n)) == ffi.ERR_INVALID_ARGUMENT
    assert lib.tcscf_schedule_items(10, 10, 1, 1, 148, None, 2, C.byref(n)) == ffi.ERR_INVALID_ARGUMENT
