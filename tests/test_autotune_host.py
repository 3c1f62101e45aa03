"""Host side of the launch-schedule autotuner (no device needed).

The autotuner measures candidate r2 split counts of the persistent tensor-core launch; which
candidates it measures is host arithmetic over the launch's tile and block counts (128 r1 rows per
tile, 64 r2 points per block), restated here independently and compared with the library's.
"""
import ctypes as C

import numpy as np
import pytest

from tcscf_b200 import ffi

BM, BK = 128, 64


def _candidates(n1, n2, sms):
    tiles = -(-n1 // BM)
    blocks = -(-n2 // BK)

    def effective(want):
        per = -(-blocks // want)
        return -(-blocks // per)

    out = [effective(max(1, min(sms // max(1, tiles), blocks // 4)))]
    for s in (1, 2, 3, 4, 6, 8):
        if s > max(1, blocks // 16):
            break
        e = effective(s)
        if e not in out:
            out.append(e)
    return out


@pytest.mark.parametrize("n, expect", [
    (406_000, [1, 2, 3, 4, 6, 8]),   # Kr: 3172 r1 tiles, more than the SMs -> default no split
    (59_000, [1, 2, 3, 4, 6, 8]),    # Ne
    (2_500, [7, 1, 2]),              # He: 20 tiles -> default 148 // 20 = 7 splits of 40 blocks
    (1_280, [5, 1]),                 # 10 tiles, 20 blocks: default 5 (blocks // 4), nothing else keeps 16 blocks
    (100, [1]),                      # one tile, two blocks
])
def test_split_candidates_at_known_sizes(n, expect):
    assert ffi.autotune_split_candidates(n, n, 148) == expect


def test_split_candidates_match_restatement():
    rng = np.random.default_rng(7)
    for _ in range(400):
        n1 = int(rng.integers(1, 2_000_000))
        n2 = int(rng.integers(1, 2_000_000))
        sms = int(rng.choice([1, 8, 132, 148, 160]))
        got = ffi.autotune_split_candidates(n1, n2, sms)
        assert got == _candidates(n1, n2, sms), (n1, n2, sms)
        blocks = -(-n2 // BK)
        assert len(set(got)) == len(got)
        for s in got[1:]:
            # every candidate beyond the default keeps at least 16 blocks of 64 points per split
            assert blocks // s >= 16 or s == 1


def test_split_candidates_capacity_and_arguments():
    lib = ffi.lib()
    buf = (C.c_int * 2)()
    n = C.c_int(-1)
    assert lib.tcscf_autotune_split_candidates(406_000, 406_000, 148, buf, 2, C.byref(n)) == ffi.OK
    assert n.value == 2 and list(buf) == [1, 2]
    assert lib.tcscf_autotune_split_candidates(406_000, 406_000, 148, None, 0, C.byref(n)) == ffi.OK and n.value == 0
    for args in [(0, 10, 148), (10, 0, 148), (10, 10, 0), (1 << 40, 10, 148)]:
        assert lib.tcscf_autotune_split_candidates(*args, buf, 2, C.byref(n)) == ffi.ERR_INVALID_ARGUMENT
    assert lib.tcscf_autotune_split_candidates(10, 10, 148, None, 2, C.byref(n)) == ffi.ERR_INVALID_ARGUMENT


def test_autotune_entry_points_reject_null_context():
    lib = ffi.lib()
    a, b, c = C.c_int(), C.c_int(), C.c_int()
    assert lib.tcscf_set_autotune(None, 1) == ffi.ERR_INVALID_ARGUMENT
    assert lib.tcscf_autotune_stats(None, C.byref(a), C.byref(b), C.byref(c)) == ffi.ERR_INVALID_ARGUMENT
