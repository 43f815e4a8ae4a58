"""Host pool generator of libnqb.so against the oracle and the reference's pool vectors.
No GPU needed: pool generation is host code."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN_DIR

GOLD = json.load(open(os.path.join(GOLDEN_DIR, "ref_vectors.json")))


@pytest.mark.parametrize("n", range(4, 15))
def test_pool_bitwise_equals_oracle(nqb, nqo, n):
    for d in range(2, n):
        got = nqb.generate_pool(n, d)
        want = nqo.pool(n, d)
        assert len(got) == len(want), (n, d)
        assert got.tobytes() == want.tobytes(), (n, d)


@pytest.mark.parametrize("n,d", [(17, 5), (18, 6), (19, 5), (21, 4), (22, 4)])
def test_pool_bitwise_equals_oracle_larger(nqb, nqo, n, d):
    assert nqb.generate_pool(n, d).tobytes() == nqo.pool(n, d).tobytes()


@pytest.mark.parametrize("case", [p for p in GOLD["pools"] if p["d"] >= 2], ids=lambda c: f"n{c['n']}d{c['d']}")
def test_pool_sizes_match_reference(nqb, case):
    assert nqb.pool_size(case["n"], case["d"]) == case["states"]
    assert nqb.pool_weighted_size(case["n"], case["d"]) == case["weighted"]


def test_pool_file_names(nqb):
    # pre_gen_state_files (test.cu:87-105): weighted pool sizes per (n, lock row)
    for f in GOLD["pool_file_sizes"]:
        if f["n"] <= 21:
            assert nqb.pool_weighted_size(f["n"], f["d"]) == f["weighted"], f


def test_alloc_variant_matches(nqb):
    a = nqb.generate_pool(13, 4)
    b = nqb.generate_pool_alloc(13, 4)
    assert a.tobytes() == b.tobytes()


def test_depth1_pool_is_row0_placements(nqb):
    for n in range(4, 16):
        p = nqb.generate_pool(n, 1)
        assert len(p) == (n + 1) // 2
        assert list(p["cols"]) == [1 << c for c in range(len(p))]
        assert all(p["row"] == 1)
        assert list(p["weight"]) == [2 if c < n // 2 else 1 for c in range(len(p))]
        assert int(p["weight"].sum()) == n


def test_weights_and_fields(nqb):
    p = nqb.generate_pool(11, 3)
    assert set(np.unique(p["weight"])) == {1, 2}
    assert all(p["n"] == 11) and all(p["row"] == 3) and all(p["flags"] == 0)
    # the middle column of an odd board carries weight 1 (GPU_NQueens.cu:356): those
    # states form the tail of the pool (row-0 column order)
    w = p["weight"]
    k = int((w == 1).sum())
    assert k > 0 and all(w[-k:] == 1) and all(w[:-k] == 2)
    assert all(nqb.generate_pool(12, 3)["weight"] == 2)


def test_ref_record_conversion(nqb, nqo):
    for n, d in [(8, 3), (13, 3), (16, 5), (20, 4)]:
        recs, sz = nqo.pool_ref_records(n, d)
        assert sz == nqb.ref_state_size(n)
        conv = nqb.states_from_ref(n, recs.tobytes())
        assert conv.tobytes() == nqo.pool(n, d).tobytes()


@pytest.mark.parametrize("n,size", [(13, 40), (19, 40), (20, 48), (22, 48), (31, 56)])
def test_ref_state_size(nqb, n, size):
    assert nqb.ref_state_size(n) == size


def test_invalid_depths(nqb):
    for n, d in [(3, 1), (32, 4), (8, 0), (8, 8), (8, 9)]:
        with pytest.raises(nqb.NQBError) as e:
            nqb.pool_size(n, d)
        assert e.value.status == nqb.E_INVALID
