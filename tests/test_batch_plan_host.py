"""The block plan of a batched field-solve launch (pb_host_plan_blocks; no GPU).

pb_batch_run shares a launch's blocks by each member's measured cost: members costing more
than the makespan T get blocks of their own, cheaper ones share blocks and run one after
another, and leftover blocks go to the member with the largest cost per block.  Checked here
over random cost mixes: every member runs, own blocks are contiguous and not shared, no block
is used twice, and the makespan (the largest per-block time under cost / blocks) stays near
the ideal (total cost / blocks).
"""
import ctypes as C

import numpy as np
import pytest

from thruster_cx_code_b200 import _lib


def _plan(work, total):
    lib = _lib.load()
    m = len(work)
    w = (C.c_int64 * m)(*[int(x) for x in work])
    first, count, packed = (C.c_int32 * m)(), (C.c_int32 * m)(), (C.c_int32 * m)()
    _lib.check(lib.pb_host_plan_blocks(w, m, total, first, count, packed), "pb_host_plan_blocks")
    return np.array(first[:]), np.array(count[:]), np.array(packed[:])


def _makespan(work, total, first, count, packed):
    per_block = np.zeros(total)
    owner = -np.ones(total, dtype=int)
    for i, (f, c, p) in enumerate(zip(first, count, packed)):
        assert 0 <= f and f + c <= total and c >= 1
        if p:
            assert c == 1
            assert owner[f] in (-1, -2), "a packed member on a block of its own member"
            owner[f] = -2
            per_block[f] += work[i]
        else:
            for q in range(f, f + c):
                assert owner[q] == -1, "a block used twice"
                owner[q] = i
                per_block[q] = work[i] / c
    return per_block.max()


def test_random_mixes():
    rng = np.random.default_rng(3)
    worst = 0.0
    for _ in range(300):
        m = int(rng.integers(1, 149))
        work = np.exp(rng.uniform(0, 6, m)) * 1000 + 1
        first, count, packed = _plan(work, 148)
        ms = _makespan(work, 148, first, count, packed)
        ideal = max(work.sum() / 148, 0.0)
        worst = max(worst, ms / ideal)
        # never worse than one member alone on a block when it costs the most
        assert ms <= work.max() * (1 + 1e-9)
    assert worst < 1.6, worst


def test_sweep_like_mix():
    """26 large, 19 medium and 19 small members: the small ones share blocks, which the large
    ones get (four or five each instead of about three)."""
    work = [80000 + 1000 * (i % 7) for i in range(26)] + [20000 + 500 * (i % 5) for i in range(19)] + \
           [4500 + 100 * (i % 3) for i in range(19)]
    first, count, packed = _plan(work, 148)
    assert packed[45:].all()
    assert (count[:26] >= 4).all()
    ms = _makespan(np.array(work, float), 148, first, count, packed)
    assert ms <= 1.2 * sum(work) / 148


def test_arguments_refused():
    lib = _lib.load()
    w = (C.c_int64 * 3)(1, 2, 3)
    o = (C.c_int32 * 3)()
    assert lib.pb_host_plan_blocks(w, 3, 2, o, o, o) != 0
    w0 = (C.c_int64 * 2)(1, 0)
    assert lib.pb_host_plan_blocks(w0, 2, 4, o, o, o) != 0
