"""Batch plans: a board set solved through a captured CUDA graph with an autotuned launch,
replayed several times.  Per-board counts must equal the oracle's (and, for the full
65,536-board set of uneven partial boards, the plain form's) exactly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def model(nqb):
    boards = nqb.sample_boards(nqb.MODEL_SEED, 40000, 14, 18, 2, 7)
    nodes, _ = nqb.record_nodes(boards)
    m = nqb.Model(seed=3)
    m.train(boards, np.log2(1.0 + nodes.astype(np.float64)).astype(np.float32), epochs=5, batch=2048, lr=2e-3)
    yield m
    m.close()


@pytest.fixture(scope="module")
def small_batch(nqb, nqo):
    boards = nqb.sample_boards(4242, 6000, 10, 14, 1, 6)
    want, nodes = nqo.solve_states(boards)
    return boards, want, nodes


@pytest.mark.parametrize("learned,autotune", [(False, False), (False, True), (True, False), (True, True)])
def test_plan_matches_oracle_over_replays(nqb, small_batch, model, learned, autotune):
    boards, want, nodes = small_batch
    plan = nqb.BatchPlan(boards, model=model if learned else None, autotune=autotune)
    cfg = plan.config()
    assert cfg["block_size"] in (64, 128, 256)
    for _ in range(3):  # graph replays start from zeroed outputs and an empty queue
        got, st = plan.run()
        assert np.array_equal(got, want)
        assert st["nodes"] == nodes
    plan.close()


def test_uneven_board_batch_full_size(nqb, nqo, model):
    """The 65,536 seeded uneven partial boards (n 16..20, depth 3..7): the learned plan (split
    and ordered queue, graph replays) against the batched form without a model (the boards as
    given, in order) and against the oracle on a subsample.  (Autotuning is covered on the
    smaller batch above; here it would only add candidate runs.)"""
    boards = nqb.sample_boards(nqb.BATCH_SEED, 65536, 16, 20, 3, 7)
    plan = nqb.BatchPlan(boards, model=model, autotune=False)
    got, st = plan.run()
    got2, _ = plan.run()
    fifo, st_fifo = nqb.solve_batch(boards, form=1)
    assert np.array_equal(got, fifo) and np.array_equal(got2, fifo)
    assert st["nodes"] == st_fifo["nodes"]
    assert st["items"] > len(boards)  # the learned schedule split the large boards
    small = np.flatnonzero((boards["n"] <= 17) & (boards["row"] >= 6))[:150]
    want, _ = nqo.solve_states(boards[small])
    assert np.array_equal(got[small], want)
    plan.close()


def test_plan_rejects_bad_boards(nqb):
    b = np.zeros(4, dtype=nqb.STATE_DTYPE)
    b["n"] = [8, 8, 40, 8]
    with pytest.raises(nqb.NQBError) as e:
        nqb.BatchPlan(b, autotune=False)
    assert e.value.status == nqb.E_INVALID
