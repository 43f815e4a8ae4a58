"""Error paths under allocation failure, through the library's test hook
(nqb_debug_fail_allocation).  Each test makes the k-th allocation of one call fail, for
k = 0, 1, ... until the call no longer reaches the failing allocation.  Every call the hook
hit must answer NQB_E_NOMEM with its outputs cleared, and the calls after it must give the
same results as a call that never failed (buffers released, no state left behind).

The reference has no such hook: its generator reports ENOMEM through errno and its solver
exits (n_queens.cu:39-41, deffinitions.cuh:148-156); the library returns status codes."""
import ctypes
import os

import numpy as np
import pytest

KAT = {13: 73712, 14: 365596, 16: 14772512, 17: 95815104}


def _status(fn):
    try:
        fn()
        return 0
    except Exception as e:  # NQBError carries the library's status
        if hasattr(e, "status"):
            return e.status
        raise


def _sweep(nqb, call, limit=256):
    """Runs `call` (returning a status) with allocation k failing, k = 0, 1, ...  Returns the
    statuses of the calls the hook hit and the status of the first call it missed."""
    hit = []
    try:
        for k in range(limit):
            nqb.debug_fail_allocation(k)
            st = call()
            left = nqb.debug_fail_allocation(-1)
            if left >= 0:  # the call made no more than k allocations: the hook never fired
                return hit, st
            hit.append(st)
    finally:
        nqb.debug_fail_allocation(-1)
    raise AssertionError(f"still allocating after {limit} allocations")


def test_hook_counts_down_and_turns_off(nqb):
    assert nqb.debug_fail_allocation(5) == -1
    assert nqb.debug_fail_allocation(-7) == 5  # replaced countdown; any negative value is off
    assert nqb.debug_fail_allocation(-1) == -1


def test_host_pool_allocation_failure(nqb):
    L = nqb.lib()
    f = L.nqb_generate_pool
    out = []

    def call():
        p = ctypes.c_void_p(1)
        c = ctypes.c_uint64(0)
        st = f(12, 4, ctypes.byref(p), ctypes.byref(c))
        out.append((st, p.value, c.value))
        if p.value:
            L.nqb_free(p)
        return st

    hit, last = _sweep(nqb, call)
    assert hit == [nqb.E_NOMEM] and last == nqb.OK
    assert out[0][1] is None  # the failed call hands back no buffer
    assert out[-1][2] == len(nqb.generate_pool(12, 4))


def test_placements_allocation_failure(nqb):
    want = nqb.generate_pool_placements(13, 5)
    hit, last = _sweep(nqb, lambda: _status(lambda: nqb.generate_pool_placements(13, 5)))
    assert hit == [nqb.E_NOMEM] and last == nqb.OK
    assert np.array_equal(nqb.generate_pool_placements(13, 5), want)


def test_state_file_reader_allocation_failure(nqb, tmp_path):
    # 200k+ boards in one segment: the reader's placement array grows several times
    pl = nqb.generate_pool_placements(16, 6)
    assert len(pl) > 3 * (1 << 16)
    path = os.path.join(tmp_path, "pool.nqsf")
    nqb.write_state_file(path, pl, 16, 6)
    info, want = nqb.read_state_file(path)
    hit, last = _sweep(nqb, lambda: _status(lambda: nqb.read_state_file(path)))
    assert len(hit) >= 3 and set(hit) == {nqb.E_NOMEM} and last == nqb.OK
    info2, got = nqb.read_state_file(path)
    assert info2 == info and np.array_equal(got, want)


def test_state_file_reader_frees_on_failure(nqb, tmp_path):
    # the raw call: a failed read leaves *placements null (nothing for the caller to free)
    L = nqb.lib()
    pl = nqb.generate_pool_placements(14, 5)
    path = os.path.join(tmp_path, "p.nqsf")
    nqb.write_state_file(path, pl, 14, 5)
    f = L.nqb_read_state_file
    info = nqb.StateFileInfo()
    p = ctypes.c_void_p(1)
    nqb.debug_fail_allocation(0)
    try:
        st = f(path.encode(), 1, 0, ctypes.byref(info), ctypes.byref(p))
    finally:
        nqb.debug_fail_allocation(-1)
    assert st == nqb.E_NOMEM and not p.value
