"""The learned cost model: features, gradients against a float64 CPU restatement, training on
solver-recorded node counts, and the exactness of learned scheduling (splitting and ordering
the batched queue must not change any count or node total)."""
import json
import os

import numpy as np
import pytest

import mlp_ref
from conftest import GOLDEN_DIR

KAT = {int(k): v for k, v in json.load(open(os.path.join(GOLDEN_DIR, "ref_vectors.json")))["kat_counts"].items()}


def test_features_match_cpu_restatement(nqb):
    boards = nqb.sample_boards(5, 500, 8, 31, 1, 7)
    got = nqb.model_features(boards)
    want = mlp_ref.features(boards)
    assert got.shape == (500, 112)
    assert np.array_equal(got, want.astype(np.float32))


def test_param_layout_constants(nqb):
    assert nqb.MODEL_PARAMS == mlp_ref.NPARAMS == 31105
    assert nqb.MODEL_INPUTS == mlp_ref.IN


@pytest.fixture(scope="module")
def model(nqb):
    m = nqb.Model(device=0, seed=7)
    yield m
    m.close()


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12))


@pytest.mark.gpu
def test_gradients_match_float64_oracle(nqb, model):
    rng = np.random.default_rng(3)
    boards = nqb.sample_boards(11, 512, 12, 20, 2, 8)
    p = model.get_params()
    p[mlp_ref.KB1:mlp_ref.KW2] = rng.normal(0, 0.1, mlp_ref.H)
    p[mlp_ref.KB2:mlp_ref.KW3] = rng.normal(0, 0.1, mlp_ref.H)
    p[mlp_ref.KB3] = 3.0
    model.set_params(p)
    t = rng.normal(10, 4, len(boards)).astype(np.float32)
    loss, g = model.loss_grad(boards, t)
    X = mlp_ref.features(boards)
    want_loss, want_g = mlp_ref.loss_grad(p.astype(np.float64), X, t.astype(np.float64))
    assert abs(loss - want_loss) <= 1e-3 * want_loss
    blocks = {"W1": (mlp_ref.KW1, mlp_ref.KB1), "b1": (mlp_ref.KB1, mlp_ref.KW2), "W2": (mlp_ref.KW2, mlp_ref.KB2),
              "b2": (mlp_ref.KB2, mlp_ref.KW3), "w3": (mlp_ref.KW3, mlp_ref.KB3), "b3": (mlp_ref.KB3, mlp_ref.NPARAMS)}
    for name, (a, b) in blocks.items():
        # FP16 operands / FP32 accumulation on the GPU against float64 with the same fp16
        # rounding points: relative L2 error of every gradient block within 1e-2
        assert _rel(g[a:b], want_g[a:b]) < 1e-2, name


@pytest.mark.gpu
def test_predict_matches_forward_oracle(nqb, model):
    boards = nqb.sample_boards(12, 3000, 8, 31, 1, 7)
    y = model.predict(boards)
    want, _ = mlp_ref.forward(model.get_params().astype(np.float64), mlp_ref.features(boards))
    assert np.max(np.abs(y - want)) < 2e-3 * max(1.0, np.max(np.abs(want)))


@pytest.mark.gpu
def test_record_nodes_matches_oracle(nqb, nqo):
    boards = nqb.sample_boards(21, 4000, 8, 14, 1, 6)
    nodes, counts = nqb.record_nodes(boards)
    want_counts, total_nodes = nqo.solve_states(boards)
    assert np.array_equal(counts, want_counts)
    assert int(nodes.sum()) == total_nodes
    for i in range(0, 4000, 397):
        c, nd = nqo.solve_states(boards[i:i + 1])
        assert int(nodes[i]) == nd


@pytest.mark.gpu
def test_training_reduces_error(nqb):
    boards = nqb.sample_boards(nqb.MODEL_SEED, 60000, 16, 16, 3, 7)
    nodes, _ = nqb.record_nodes(boards)
    t = np.log2(1.0 + nodes.astype(np.float64)).astype(np.float32)
    tr, va = slice(0, 54000), slice(54000, 60000)
    m = nqb.Model(seed=1)
    losses = m.train(boards[tr], t[tr], epochs=6, batch=2048, lr=2e-3)
    assert losses[-1] < losses[0]
    pred = m.predict(boards[va])
    rmse = float(np.sqrt(np.mean((pred - t[va]) ** 2)))
    base = float(np.sqrt(np.mean((t[va] - t[tr].mean()) ** 2)))
    assert rmse < 0.6 * base, (rmse, base)
    m.close()


@pytest.fixture(scope="module")
def trained(nqb):
    boards = nqb.sample_boards(nqb.MODEL_SEED, 40000, 14, 18, 2, 7)
    nodes, _ = nqb.record_nodes(boards)
    m = nqb.Model(seed=2)
    m.train(boards, np.log2(1.0 + nodes.astype(np.float64)).astype(np.float32), epochs=5, batch=2048, lr=2e-3)
    yield m
    m.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n,d", [(12, 2), (14, 3), (16, 2), (17, 3), (18, 4)])
def test_learned_schedule_is_exact(nqb, trained, n, d):
    c0, st0 = nqb.count_ex(n, d, form=1)
    c1, st1 = nqb.count_ex(n, d, form=1, model=trained)
    assert c1 == c0 == KAT[n]
    assert st1["nodes"] == st0["nodes"]


@pytest.mark.gpu
def test_learned_schedule_per_board(nqb, nqo, trained):
    boards = nqb.sample_boards(31, 3000, 10, 16, 1, 5)
    got, st = nqb.solve_batch(boards, form=1, model=trained)
    want, nodes = nqo.solve_states(boards)
    assert np.array_equal(got, want)
    assert st["nodes"] == nodes


@pytest.mark.gpu
def test_schedule_ablation_arms_are_exact(nqb, trained):
    """Ablation of the learned schedule: the same split-and-order pipeline driven by the trained
    network, an untrained one and the two model-free costs, against FIFO with work stealing.
    N=17 with a depth-3 pool has 1,473 items for ~150k resident lanes.  Every arm must be
    exact; the arms' speeds are measured by the bench (extras.ablation), and here the trained
    arm must at least not lose to the untrained network by more than noise."""
    untrained = nqb.Model(seed=5)
    try:
        arms = {"fifo": {}, "untrained": {"model": untrained}, "free_x_rows": {"sched_cost": 1},
                "lookahead": {"sched_cost": 2}, "trained": {"model": trained}}
        ms = {}
        for name, kw in arms.items():
            for _ in range(2):  # the second run is the measured one
                c, st = nqb.count_ex(17, 3, form=1, **kw)
            assert c == KAT[17], name
            ms[name] = st["kernel_ms"]
            if name != "fifo":
                assert st["items"] > 1473, name
        assert ms["trained"] < 1.5 * ms["untrained"] + 5.0, ms
    finally:
        untrained.close()


@pytest.mark.gpu
def test_no_split_rounds_still_exact(nqb, trained):
    c, st = nqb.count_ex(15, 2, form=1, model=trained, max_split_rounds=0)
    assert c == KAT[15]


@pytest.mark.gpu
def test_predict_many_tiles(nqb, model):
    """Enough boards for several 128-row tiles per persistent block (the completion barrier
    changes phase twice per tile), checked row by row against the CPU forward pass."""
    boards = nqb.sample_boards(77, 200_000, 8, 22, 1, 7)
    y = model.predict(boards)
    want, _ = mlp_ref.forward(model.get_params().astype(np.float64), mlp_ref.features(boards))
    assert np.max(np.abs(y - want)) < 2e-3 * max(1.0, np.max(np.abs(want)))
    assert np.array_equal(model.predict(boards[:1]), y[:1])  # a single, partial tile


@pytest.mark.gpu
def test_predict_wait_timeout_reports_stall_and_recovers(nqb, model):
    """Failure detection without a fault: a one-iteration bound on the tensor-core completion
    wait runs out, the kernel drains its products in flight, frees its tensor memory and the
    call returns E_STALL; the next calls on the same model and device are exact again."""
    boards = nqb.sample_boards(91, 50_000, 10, 20, 2, 6)
    want = model.predict(boards)
    with pytest.raises(nqb.NQBError) as e:
        model.predict(boards, wait_limit=1)
    assert e.value.status == nqb.E_STALL
    assert np.array_equal(model.predict(boards), want)
    assert nqb.count(14, 4, form=1, model=model) == 365596
