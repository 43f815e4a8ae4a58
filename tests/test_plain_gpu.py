"""Parity of the plain form (one thread per state) on the GPU, through the C ABI, against the
reference's vectors (tests/golden) and the oracle.  Bit-exact: counts, nodes, unit nodes."""
import ctypes
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN_DIR

pytestmark = pytest.mark.gpu
GOLD = json.load(open(os.path.join(GOLDEN_DIR, "ref_vectors.json")))
KAT = {int(k): v for k, v in GOLD["kat_counts"].items()}
FULL_REPLAYS = [r for r in GOLD["replays"] if r["stride"] == 1 and r["d"] >= 2]
SAMPLED_REPLAYS = [r for r in GOLD["replays"] if r["stride"] > 1]


def test_config1_n13_d3(nqb):
    c, st = nqb.count_ex(13, 3, count_unit_nodes=True)
    assert c == 73712
    assert st["states"] == 553 and st["nodes"] == 2531097 and st["unit_nodes"] == 935892


@pytest.mark.parametrize("case", FULL_REPLAYS, ids=lambda c: f"n{c['n']}d{c['d']}")
def test_full_pool_matches_reference_replay(nqb, case):
    c, st = nqb.count_ex(case["n"], case["d"], count_unit_nodes=True)
    assert c == case["count"] == KAT[case["n"]]
    assert st["nodes"] == case["nodes"]
    assert st["unit_nodes"] == case["unit"]
    c2, st2 = nqb.count_ex(case["n"], case["d"])  # production kernel (no unit counting)
    assert c2 == c and st2["nodes"] == case["nodes"]


@pytest.mark.parametrize("case", SAMPLED_REPLAYS, ids=lambda c: f"n{c['n']}d{c['d']}s{c['stride']}")
def test_pool_sample_matches_reference_replay(nqb, case):
    pool = nqb.generate_pool(case["n"], case["d"])
    assert len(pool) == case["states"]
    sample = pool[case["offset"]::case["stride"]]
    assert len(sample) == case["sampled"]
    total, st = nqb.solve_states(sample, count_unit_nodes=True)
    assert total == case["count"]
    assert st["nodes"] == case["nodes"]
    assert st["unit_nodes"] == case["unit"]


@pytest.mark.parametrize("n,d", [(8, 2), (10, 5), (14, 4), (15, 6), (16, 4), (17, 5), (18, 6)])
def test_kat_counts(nqb, n, d):
    assert nqb.count(n, d) == KAT[n]


@pytest.mark.parametrize("block", [64, 128, 256])
def test_block_sizes_agree(nqb, block):
    assert nqb.count(15, 5, block_size=block) == KAT[15]


def test_depth1_pool_counts_correctly(nqb):
    # The library's depth-1 pool is the row-0 placements (the reference's is not; see
    # tests/test_oracle.py::test_reference_depth1_pool_quirk).
    for n in range(6, 13):
        assert nqb.count(n, 1) == KAT[n]


def test_deep_pools(nqb):
    for n in (8, 11, 13):
        assert nqb.count(n, n - 1) == KAT[n]
        assert nqb.count(n, n - 2) == KAT[n]


def test_reference_records_drop_in(nqb, nqo):
    for n, d in [(12, 4), (14, 5), (16, 5)]:
        recs, _ = nqo.pool_ref_records(n, d)
        assert nqb.solve_ref_states(n, recs.tobytes(), d) == KAT[n]


def test_reference_records_wrong_lock_row(nqb, nqo):
    recs, _ = nqo.pool_ref_records(12, 4)
    with pytest.raises(nqb.NQBError) as e:
        nqb.solve_ref_states(12, recs.tobytes(), 5)
    assert e.value.status == nqb.E_INVALID


def test_mixed_board_batch_matches_oracle(nqb, nqo):
    boards = nqb.sample_boards(12345, 3000, 8, 14, 1, 6)
    got, st = nqb.solve_batch(boards)
    want, nodes = nqo.solve_states(boards)
    assert np.array_equal(got, want)
    assert st["nodes"] == nodes


def test_batch_edge_cases(nqb, nqo):
    b = np.zeros(6, dtype=nqb.STATE_DTYPE)
    b["n"] = [8, 8, 10, 31, 5, 4]
    b["weight"] = [1, 3, 1, 0, 1, 1]
    # board 1: a full 8-queens solution handed in (counts once, weight 3)
    sol = [0, 4, 7, 5, 2, 6, 1, 3]
    cols = ld = rd = 0
    for c in sol:
        bb = 1 << c
        cols |= bb
        ld = ((ld | bb) << 1) & 0xFFFFFFFF
        rd = (rd | bb) >> 1
    b[1] = (cols, ld, rd, 8, 8, 3, 0)
    # board 2: next row dead -> 0
    b[2] = (0b11, 0b1111111100, 0, 2, 10, 1, 0)
    # board 3: weight 0 on a big board with a single free column left
    b[3] = (0x7FFFFFFF & ~1, 0, 0, 30, 31, 0, 0)
    got, _ = nqb.solve_batch(b)
    want, _ = nqo.solve_states(b)
    assert list(got) == list(want)
    assert got[0] == 92 and got[1] == 3 and got[2] == 0 and got[3] == 0 and got[4] == 10 and got[5] == 2


def test_empty_inputs(nqb):
    t, st = nqb.solve_states(np.zeros(0, dtype=nqb.STATE_DTYPE))
    assert t == 0
    out, _ = nqb.solve_batch(np.zeros(0, dtype=nqb.STATE_DTYPE))
    assert len(out) == 0


def test_device_resident_launch_and_stack_check(nqb):
    torch = pytest.importorskip("torch")
    pool = nqb.generate_pool(14, 4)
    d_states = torch.from_numpy(pool.view(np.uint8).copy()).cuda()
    d_out = torch.zeros(4, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    nqb.plain_launch(d_states.data_ptr(), len(pool), d_out.data_ptr(), stack_depth=14 - 4 - 1, stream=s)
    torch.cuda.synchronize()
    out = d_out.cpu().numpy().astype(np.uint64)
    assert out[0] == KAT[14] and out[3] == 0
    # a stack that is too shallow is reported through the error word, not by a fault
    d_out.zero_()
    nqb.plain_launch(d_states.data_ptr(), len(pool), d_out.data_ptr(), stack_depth=2, stream=s)
    torch.cuda.synchronize()
    assert int(d_out[3].item()) & 1 == 1


def test_count_17_5_config2(nqb):
    c, st = nqb.count_ex(17, 5)
    assert c == 95815104
    assert st["states"] == 114434 and st["nodes"] == 4275902721


@pytest.mark.parametrize("n", [4, 8, 11, 13, 16, 19])
def test_device_pool_equals_host_pool(nqb, n):
    depths = {1, 2, n // 2, n - 2, n - 1} if n <= 16 else {1, 2, 5, 7, 9}  # deep N=19 pools hold billions
    for d in sorted(depths):
        if 1 <= d < n:
            assert nqb.generate_pool_device(n, d).tobytes() == nqb.generate_pool(n, d).tobytes(), (n, d)


def test_device_pool_large(nqb):
    p = nqb.generate_pool_device(21, 7)
    assert len(p) == 39430182 and int(p["weight"].sum()) == 75580634
    h = nqb.generate_pool(21, 7)
    assert p.tobytes() == h.tobytes()


@pytest.mark.parametrize("form", [0, 1])
def test_count_with_host_or_device_pool(nqb, form):
    for n, d in [(12, 3), (16, 5), (17, 4)]:
        c_dev, s_dev = nqb.count_ex(n, d, form=form)
        c_host, s_host = nqb.count_ex(n, d, form=form, host_pool=True)
        assert c_dev == c_host == KAT[n] and s_dev["nodes"] == s_host["nodes"]
        assert s_dev["h2d_ms"] == 0.0 and s_dev["states"] == s_host["states"]


@pytest.mark.parametrize("devices", [[0], [0, 0], [0, 0, 0]])
def test_solve_states_multi_slices(nqb, devices):
    pool = nqb.generate_pool(15, 5)
    total, st = nqb.solve_states_multi(pool, devices, form=1)
    one, st1 = nqb.solve_states_multi(pool, [0])
    assert total == one == KAT[15] and st["nodes"] == st1["nodes"] and st["states"] == len(pool)
    assert nqb.device_count() >= 1
    # fewer states than devices: the first slices are empty, the last takes them all
    t, _ = nqb.solve_states_multi(pool[:2], devices)
    w, _ = nqb.solve_states(pool[:2])
    assert t == w


def test_cached_device_memory_reused_and_trimmed(nqb):
    """Repeated calls reuse the library's cached device memory; trimming returns it and
    the next call maps it again, with the same result."""
    for _ in range(3):
        assert nqb.count(16, 5, form=1) == KAT[16]
    nqb.trim_device_memory(0)
    assert nqb.count(16, 5) == KAT[16]
    nqb.trim_device_memory(0)
    with pytest.raises(nqb.NQBError):
        nqb.trim_device_memory(-1)


def test_int32_peak_microbenchmark(nqb):
    """The roofline denominator: every kind runs, and the best is within the issue limit
    (one warp instruction per SM sub-partition per clock at the maximum SM clock)."""
    best, kinds = nqb.measure_int32_peak(0)
    assert set(kinds) == {"lop3", "add", "imad", "lop3_imad"} and all(v > 1e12 for v in kinds.values())
    assert best == max(kinds.values()) and best <= 148 * 4 * 32 * 2.0e9 * 1.02
