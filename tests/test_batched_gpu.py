"""Parity of the batched form (persistent kernel, device work queue, intra-warp re-splitting)
against the reference's vectors and the oracle.  Bit-exact counts and nodes: moving work
between lanes must neither lose nor repeat a placement."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN_DIR

pytestmark = pytest.mark.gpu
GOLD = json.load(open(os.path.join(GOLDEN_DIR, "ref_vectors.json")))
KAT = {int(k): v for k, v in GOLD["kat_counts"].items()}
B = dict(form=1)


@pytest.mark.parametrize("case", [r for r in GOLD["replays"] if r["stride"] == 1 and r["d"] >= 2],
                         ids=lambda c: f"n{c['n']}d{c['d']}")
def test_full_pool_matches_reference_replay(nqb, case):
    c, st = nqb.count_ex(case["n"], case["d"], **B)
    assert c == case["count"] == KAT[case["n"]]
    assert st["nodes"] == case["nodes"]


@pytest.mark.parametrize("case", [r for r in GOLD["replays"] if r["stride"] > 1],
                         ids=lambda c: f"n{c['n']}d{c['d']}s{c['stride']}")
def test_pool_sample_matches_reference_replay(nqb, case):
    pool = nqb.generate_pool(case["n"], case["d"])
    sample = pool[case["offset"]::case["stride"]]
    total, st = nqb.solve_states(sample, **B)
    assert total == case["count"] and st["nodes"] == case["nodes"]


@pytest.mark.parametrize("n,d", [(8, 1), (12, 1), (16, 2), (17, 3), (18, 4), (19, 7)])
def test_counts_few_large_items(nqb, n, d):
    # few, large items: the queue empties at once and the work is spread by re-splitting
    assert nqb.count(n, d, **B) == KAT[n]


@pytest.mark.parametrize("block", [64, 128, 256])
def test_block_sizes(nqb, block):
    assert nqb.count(16, 3, block_size=block, **B) == KAT[16]


def test_per_board_counts_match_oracle(nqb, nqo):
    boards = nqb.sample_boards(777, 5000, 8, 15, 1, 7)
    got, st = nqb.solve_batch(boards, **B)
    want, nodes = nqo.solve_states(boards)
    assert np.array_equal(got, want)
    assert st["nodes"] == nodes


def test_per_board_uneven_sizes(nqb, nqo):
    # a few empty boards (huge subtrees) among many nearly full ones
    small = nqb.sample_boards(99, 2000, 10, 12, 6, 9)
    big = np.zeros(3, dtype=nqb.STATE_DTYPE)
    big["n"] = [13, 12, 14]
    big["weight"] = 1
    boards = np.concatenate([small[:1000], big, small[1000:]])
    got, _ = nqb.solve_batch(boards, **B)
    want, _ = nqo.solve_states(boards)
    assert np.array_equal(got, want)
    assert got[1000] == KAT[13] and got[1002] == KAT[14]


def test_edge_boards(nqb, nqo):
    b = np.zeros(5, dtype=nqb.STATE_DTYPE)
    b["n"] = [8, 10, 31, 5, 4]
    b["weight"] = [1, 1, 0, 2, 1]
    b[1] = (0b11, 0b1111111100, 0, 2, 10, 1, 0)       # dead next row
    b[2] = (0x7FFFFFFF & ~1, 0, 0, 30, 31, 0, 0)      # one free column, weight 0
    got, _ = nqb.solve_batch(b, **B)
    assert list(got) == [92, 0, 0, 20, 2]


def test_device_resident_launch_with_order(nqb):
    torch = pytest.importorskip("torch")
    pool = nqb.generate_pool(15, 4)
    d_items = torch.from_numpy(pool.view(np.uint8).copy()).cuda()
    order = torch.randperm(len(pool), generator=torch.Generator().manual_seed(3)).to(torch.int32).cuda()
    d_head = torch.zeros(1, dtype=torch.int32, device="cuda")
    d_out = torch.zeros(4, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    nqb.batched_launch(d_items.data_ptr(), len(pool), d_head.data_ptr(), d_out.data_ptr(),
                       d_order_ptr=order.data_ptr(), stack_depth=15 - 4 - 1, stream=s)
    torch.cuda.synchronize()
    assert int(d_out[0].item()) == KAT[15] and int(d_out[3].item()) == 0
    assert int(d_head.item()) >= len(pool)


def _launch_ex(nqb, torch, boards, **kw):
    """One nqb_batched_launch_ex on device copies of `boards`; returns the four result words."""
    d_items = torch.from_numpy(boards.view(np.uint8).copy()).cuda()
    scratch = torch.zeros(kw.pop("scratch_bytes", nqb.BATCHED_SCRATCH_BYTES), dtype=torch.uint8, device="cuda")
    d_out = torch.zeros(4, dtype=torch.int64, device="cuda")
    d_lanes = kw.pop("lanes", None)
    s = torch.cuda.current_stream().cuda_stream
    nqb.batched_launch_ex(d_items.data_ptr(), len(boards), scratch.data_ptr(), scratch.numel(), d_out.data_ptr(),
                          d_lane_stats_ptr=d_lanes.data_ptr() if d_lanes is not None else None,
                          stack_depth=int(max(b["n"] for b in boards)), stream=s, **kw)
    torch.cuda.synchronize()
    return [int(x) for x in d_out.cpu().numpy().astype(np.uint64)]


def test_steal_ring_launch_matches_oracle(nqb, nqo):
    # a few empty boards (long subtrees) among small ones: the hungry warps live off the ring
    torch = pytest.importorskip("torch")
    small = nqb.sample_boards(4242, 3000, 9, 13, 2, 8)
    big = np.zeros(4, dtype=nqb.STATE_DTYPE)
    big["n"] = [14, 13, 15, 12]
    big["weight"] = 1
    boards = np.concatenate([big[:2], small, big[2:]])
    want, nodes = nqo.solve_states(boards)
    out = _launch_ex(nqb, torch, boards)
    assert out[3] == 0
    assert out[0] == int(np.sum(want)) and out[1] == nodes


@pytest.mark.parametrize("scratch_bytes", [4, 64 + 2 * 32, 64 + 32 * 1024])
def test_steal_ring_sizes(nqb, scratch_bytes):
    # no ring (the head alone), the smallest ring, and a ring that fills up and wraps laps
    torch = pytest.importorskip("torch")
    boards = np.zeros(2, dtype=nqb.STATE_DTYPE)
    boards["n"] = [15, 14]
    boards["weight"] = 1
    out = _launch_ex(nqb, torch, boards, scratch_bytes=scratch_bytes)
    assert out[3] == 0 and out[0] == KAT[15] + KAT[14]


def test_steal_wait_limit_reports_stall_then_recovers(nqb):
    # One large board: every other warp goes hungry at once and waits on the ring.  With a
    # wait bound of one poll some warp gives up, the launch reports a stall (error bit 4) and
    # nothing hangs; the next launch, with the default bound, is exact.
    torch = pytest.importorskip("torch")
    board = np.zeros(1, dtype=nqb.STATE_DTYPE)
    board["n"] = 16
    board["weight"] = 1
    out = _launch_ex(nqb, torch, board, wait_limit=1)
    assert out[3] & 4
    out = _launch_ex(nqb, torch, board)
    assert out[3] == 0 and out[0] == KAT[16]
    assert nqb.count(17, 3, **B) == KAT[17]


@pytest.mark.parametrize("n,d", [(16, 4), (17, 5), (18, 6)])
def test_lane_efficiency_counters(nqb, n, d):
    # the instrumented kernels leave counts and nodes unchanged; on pools that fill the GPU
    # the batched form keeps its lanes busier than the plain form (a pool of a few thousand
    # short items is mostly ramp-up and tail, where both forms leave lanes idle)
    eff = {}
    for form in (0, 1):
        c, st = nqb.count_ex(n, d, form=form, count_lane_steps=True)
        c0, st0 = nqb.count_ex(n, d, form=form)
        assert c == c0 == KAT[n] and st["nodes"] == st0["nodes"]
        assert 0 < st["placed_lane_steps"] <= st["lane_step_slots"]
        assert st0["lane_step_slots"] == 0
        eff[form] = st["lane_efficiency"]
    if n >= 17:
        assert eff[1] > eff[0], eff


def test_lane_counters_through_launch_ex(nqb):
    torch = pytest.importorskip("torch")
    pool = nqb.generate_pool(15, 4)
    lanes = torch.zeros(2, dtype=torch.int64, device="cuda")
    out = _launch_ex(nqb, torch, pool, lanes=lanes)
    placed, slots = (int(x) for x in lanes.cpu().numpy())
    assert out[3] == 0 and out[0] == KAT[15]
    assert 0 < placed <= slots and slots % (32 * 16) == 0
