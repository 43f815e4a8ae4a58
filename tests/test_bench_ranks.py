"""The bench's multi-rank host logic on CPU: two gloo ranks, as `torchrun --nproc-per-node 2`
would start them.  The path shards into independent replicas, so the only collective is
the max of the per-rank step times; the whole-job rate is every rank's units over that
max.  The reference arm runs on rank 0 only."""
import json
import multiprocessing as mp
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    from datetime import timedelta

    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    try:
        r, w, _ = bench.rank_env()
        ms = 1000.0 + 250.0 * r               # rank 1 is the slow one
        got = bench.max_over_ranks(ms, w)
        rate = bench.replica_rate(10 ** 12, w, got / 1e3)
        q.put((r, w, got, rate))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [x[:3] for x in res] == [(0, 2, 1250.0), (1, 2, 1250.0)]
    assert all(x[3] == pytest.approx(2 * 10 ** 12 / 1.25) for x in res)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.replica_rate(100, 1, 2.0) == 50.0


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       capture_output=True, text=True, env=env, timeout=120, cwd=ROOT)
    assert p.returncode == 0 and p.stdout.strip() == ""


def test_reference_arm_line_on_rank_zero():
    """A short reference-arm run: one JSON line with the keys the driver reads."""
    if not os.access(os.path.join(ROOT, "oracle", "_ref", "N16", "ref_harness"), os.X_OK):
        pytest.skip("oracle/_ref is not built")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1", "--n", "16", "--depth", "5", "--ref-step-seconds", "0.5",
                        "--ref-cuda", "0"],
                       capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert p.returncode == 0, p.stderr
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "nodes/s" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["e2e"]["h2d_bytes_per_step"] == 0
