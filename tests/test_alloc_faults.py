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


# ---- device paths: pools, launches, schedules, plans, the tuner and the cost model ----


@pytest.mark.gpu
@pytest.mark.parametrize("form,host_pool", [(0, False), (1, False), (0, True), (1, True)])
def test_count_allocation_failure(nqb, form, host_pool):
    c0, st0 = nqb.count_ex(14, 4, form=form, host_pool=host_pool)
    hit, last = _sweep(nqb, lambda: _status(lambda: nqb.count_ex(14, 4, form=form, host_pool=host_pool)))
    assert hit and set(hit) == {nqb.E_NOMEM} and last == nqb.OK
    c, st = nqb.count_ex(14, 4, form=form, host_pool=host_pool)
    assert c == c0 == KAT[14] and st["nodes"] == st0["nodes"]


@pytest.mark.gpu
def test_autotuned_count_allocation_failure(nqb):
    hit, last = _sweep(nqb, lambda: _status(lambda: nqb.count_ex(14, 4, autotune=True)))
    assert len(hit) >= 3 and set(hit) == {nqb.E_NOMEM} and last == nqb.OK
    assert nqb.count_ex(14, 4, autotune=True)[0] == KAT[14]


@pytest.mark.gpu
@pytest.mark.parametrize("sched_cost", [0, 2])
def test_batch_allocation_failure(nqb, sched_cost):
    boards = nqb.sample_boards(77, 2000, 10, 14, 2, 5)
    want, _ = nqb.solve_batch(boards, form=nqb.FORM_BATCHED, sched_cost=sched_cost)
    hit, last = _sweep(nqb, lambda: _status(
        lambda: nqb.solve_batch(boards, form=nqb.FORM_BATCHED, sched_cost=sched_cost)))
    assert hit and set(hit) == {nqb.E_NOMEM} and last == nqb.OK
    got, _ = nqb.solve_batch(boards, form=nqb.FORM_BATCHED, sched_cost=sched_cost)
    assert np.array_equal(got, want)


@pytest.mark.gpu
def test_plan_allocation_failure(nqb):
    boards = nqb.sample_boards(78, 3000, 10, 14, 2, 5)
    want, _ = nqb.solve_batch(boards, form=nqb.FORM_BATCHED)

    def create_and_run():
        try:
            plan = nqb.BatchPlan(boards, autotune=True, sched_cost=2)
        except nqb.NQBError as e:
            return e.status
        try:
            got, _ = plan.run()
        finally:
            plan.close()
        assert np.array_equal(got, want)
        return nqb.OK

    hit, last = _sweep(nqb, create_and_run)
    assert len(hit) >= 6 and set(hit) == {nqb.E_NOMEM} and last == nqb.OK
    assert create_and_run() == nqb.OK


@pytest.mark.gpu
def test_tuner_allocation_failure(nqb):
    hit, last = _sweep(nqb, lambda: _status(lambda: nqb.tune_count(14, [3, 4], sample_div=4)))
    assert len(hit) >= 3 and set(hit) == {nqb.E_NOMEM} and last == nqb.OK


@pytest.mark.gpu
def test_model_allocation_failure(nqb):
    boards = nqb.sample_boards(79, 512, 10, 13, 2, 5)
    targets = np.linspace(1.0, 9.0, len(boards)).astype(np.float32)

    def create():
        try:
            nqb.Model(device=0, seed=1).close()
        except nqb.NQBError as e:
            return e.status
        return nqb.OK

    hit, last = _sweep(nqb, create)
    assert len(hit) == 6 and set(hit) == {nqb.E_NOMEM} and last == nqb.OK
    m = nqb.Model(device=0, seed=1)
    try:
        hit, last = _sweep(nqb, lambda: _status(lambda: m.train(boards, targets, epochs=1, batch=256)))
        assert len(hit) >= 10 and set(hit) == {nqb.E_NOMEM} and last == nqb.OK
        p0 = m.predict(boards)
        hit, last = _sweep(nqb, lambda: _status(lambda: m.predict(boards)))
        assert len(hit) >= 3 and set(hit) == {nqb.E_NOMEM} and last == nqb.OK
        assert np.array_equal(m.predict(boards), p0)
    finally:
        m.close()
