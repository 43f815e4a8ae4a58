"""Per-board parity of the uneven partial-board batch against the reference itself: 65,536
boards, n uniform in 16..20, depth uniform in 3..7, seed 0x4E51554545534231.

tests/golden/uneven_boards.json holds a stratified sample of the batch -- every (n, depth)
cell's largest board and 7 more -- with the completions and placements that the reference's
own locked_advance_nq_state (n_queens.cu:423-445) streams from each board, mirror weighting
off (tests/golden/make_uneven_golden.py).  The CPU tests pin the fixture to the library's
board sampler; the GPU tests require the plain form, the batched form (FIFO, with work
stealing across warps) and the learned plan of the whole batch to give the same per-board
counts and nodes."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN_DIR

FIX = json.load(open(os.path.join(GOLDEN_DIR, "uneven_boards.json")))


def fixture_states(nqb):
    b = FIX["boards"]
    st = np.zeros(len(b), dtype=nqb.STATE_DTYPE)
    st["cols"] = [x["masks"][0] for x in b]
    st["ldiag"] = [x["masks"][1] for x in b]
    st["rdiag"] = [x["masks"][2] for x in b]
    st["row"] = [x["d"] for x in b]
    st["n"] = [x["n"] for x in b]
    st["weight"] = 1
    return st


def test_fixture_boards_are_the_sampled_ones(nqb):
    batch = nqb.sample_boards(FIX["seed"], FIX["count"], *FIX["n"], *FIX["depth"])
    assert FIX["seed"] == nqb.BATCH_SEED and FIX["count"] == 65536
    idx = np.array([x["index"] for x in FIX["boards"]])
    assert np.array_equal(batch[idx], fixture_states(nqb))
    for x in FIX["boards"]:  # the queen columns rebuild the masks
        cols = ld = rd = 0
        for c in x["cols"]:
            b = 1 << c
            cols, ld, rd = cols | b, ((ld | b) << 1) & 0xFFFFFFFF, (rd | b) >> 1
        assert [cols, ld, rd] == x["masks"] and len(x["cols"]) == x["d"]


def test_fixture_covers_every_cell():
    cells = {(x["n"], x["d"]) for x in FIX["boards"]}
    assert cells == {(n, d) for n in range(16, 21) for d in range(3, 8)}
    for cell in cells:
        assert sum((x["n"], x["d"]) == cell for x in FIX["boards"]) >= 8


def test_oracle_agrees_on_small_fixture_boards(nqb, nqo):
    st = fixture_states(nqb)
    small = [i for i, x in enumerate(FIX["boards"]) if x["nodes"] < 3_000_000]
    got, nodes = nqo.solve_states(st[small])
    assert list(got) == [FIX["boards"][i]["count"] for i in small]
    assert nodes == sum(FIX["boards"][i]["nodes"] for i in small)


@pytest.mark.gpu
@pytest.mark.parametrize("form", [0, 1], ids=["plain", "batched"])
def test_forms_match_reference_per_board(nqb, form):
    st = fixture_states(nqb)
    got, stats = nqb.solve_batch(st, form=form)
    assert list(got) == [x["count"] for x in FIX["boards"]]
    assert stats["nodes"] == sum(x["nodes"] for x in FIX["boards"])


@pytest.mark.gpu
def test_batched_per_board_nodes_match_reference(nqb):
    nodes, counts = nqb.record_nodes(fixture_states(nqb))
    assert list(nodes) == [x["nodes"] for x in FIX["boards"]]
    assert list(counts) == [x["count"] for x in FIX["boards"]]


@pytest.mark.gpu
def test_whole_batch_plans_match_reference_per_board(nqb):
    """The full 65,536-board batch, FIFO and through plans driven by a model-free cost and by a
    small trained network: the fixture's boards must come out exactly as the reference's."""
    batch = nqb.sample_boards(FIX["seed"], FIX["count"], *FIX["n"], *FIX["depth"])
    idx = np.array([x["index"] for x in FIX["boards"]])
    want = np.array([x["count"] for x in FIX["boards"]], dtype=np.uint64)
    fifo, st_f = nqb.solve_batch(batch, form=1)
    assert np.array_equal(fifo[idx], want)
    train = nqb.sample_boards(nqb.MODEL_SEED, 20000, 16, 18, 4, 8)
    tn, _ = nqb.record_nodes(train)
    model = nqb.Model(seed=3)
    model.train(train, np.log2(1.0 + tn.astype(np.float64)).astype(np.float32), epochs=3, batch=2048, lr=2e-3)
    try:
        for kw in ({"sched_cost": 2}, {"model": model}):
            plan = nqb.BatchPlan(batch, autotune=False, **kw)
            got, st_p = plan.run()
            plan.close()
            assert np.array_equal(got[idx], want), kw
            assert np.array_equal(got, fifo) and st_p["nodes"] == st_f["nodes"], kw
    finally:
        model.close()
