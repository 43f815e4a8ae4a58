"""The launch autotuner: candidates timed on a stride sample of each depth's pool agree on
the sample's count, the pick is the fastest of them, and a count run with autotuning is
exact."""
import json
import os

import pytest

from conftest import GOLDEN_DIR

pytestmark = pytest.mark.gpu
KAT = {int(k): v for k, v in json.load(open(os.path.join(GOLDEN_DIR, "ref_vectors.json")))["kat_counts"].items()}


def test_tune_over_depths_forms_and_blocks(nqb):
    r = nqb.tune_count(17, [4, 5, 6], sample_div=16)
    assert len(r["tried"]) == 3 * 6
    assert {(t["depth"], t["form"], t["block_size"]) for t in r["tried"]} == {
        (d, f, b) for d in (4, 5, 6) for f in (0, 1) for b in (64, 128, 256)}
    best = min(r["tried"], key=lambda t: t["ms"])
    assert (r["depth"], r["form"], r["block_size"]) == (best["depth"], best["form"], best["block_size"])
    assert r["sample_states"] == -(-nqb.pool_size(17, r["depth"]) // 16)


def test_tune_with_model_tries_split_factors(nqb):
    boards = nqb.sample_boards(nqb.MODEL_SEED, 20000, 14, 17, 2, 6)
    nodes, _ = nqb.record_nodes(boards)
    import numpy as np
    m = nqb.Model(seed=2)
    m.train(boards, np.log2(1.0 + nodes.astype(np.float64)).astype(np.float32), epochs=3, batch=2048, lr=2e-3)
    r = nqb.tune_count(16, [4], sample_div=4, model=m)
    assert {t["split_factor"] for t in r["tried"] if t["form"] == 1} == {1, 4, 16}
    assert len(r["tried"]) == 3 + 9
    m.close()


@pytest.mark.parametrize("n,d", [(15, 4), (17, 5)])
def test_count_with_autotune_is_exact(nqb, n, d):
    c, st = nqb.count_ex(n, d, autotune=True)
    assert c == KAT[n] and st["block_size"] in (64, 128, 256) and st["form"] in (0, 1)


def test_tune_rejects_bad_arguments(nqb):
    for args in [(17, [17]), (17, [0]), (3, [1])]:
        with pytest.raises(nqb.NQBError) as e:
            nqb.tune_count(*args)
        assert e.value.status == nqb.E_INVALID
    with pytest.raises(nqb.NQBError):
        nqb.tune_count(17, [5], sample_div=0)
