#!/usr/bin/env python
"""Benchmark: full N-Queens count N=21 (pregen depth 7) on one B200.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl nqb|reference]

One step = one full count: every state of the depth-7 pool searched to the last row.
`value` is search nodes/s with the pool already resident in HBM (kernel time by CUDA
events on the launching stream); `e2e` is the same metric through the public C ABI
call nqb_count_ex(21, 7) with host buffers: pool generation (on the GPU, seeded from the
host), kernel and result read-back inside the timed region; the reference's way (pool built
on the host and copied over, `host_pool`) is timed once beside it.  Prints one JSON line on rank 0.

`--impl reference` times the reference's own CPU path (oracle/_ref, built from the
reference's sources) on bounded stride samples of the same pool with every host core,
and, for comparison, the reference CUDA build on the same GPU.

Multi-GPU: the count runs on one GPU, so N > 1 runs N independent replicas (weak
scaling, no collective on the data path); the step time is the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

KAT = {13: 73712, 17: 95815104, 18: 666090624, 19: 4968057848, 20: 39029188884, 21: 314666222712,
       22: 2691008701644}
# Search nodes of full counts: (17, 5) and (18, 6) equal the reference's own kernel-loop
# replay (tests/golden); the others are the counts both kernel forms report, which the
# GPU tests pin on stride samples of each pool against the reference replay.
NODES = {(17, 5): 4275902721, (18, 6): 29681542262, (19, 7): 245072203329, (20, 7): 1884962763151,
         (21, 7): 16976718185320}
INT_OPS_PER_NODE = 15  # algorithmic INT32 lane-ops per node (fixed convention)
METRIC = "N=21 count wall-time & nodes/s on 1 GPU: batched+learned vs plain, bit-exact"


def load_pkg():
    from __graft_entry__ import _import_pkg
    return _import_pkg()


def rank_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(x, world, device=None):
    """The maximum of a per-rank time over all ranks (an all-reduce MAX of one value): a
    CUDA tensor on `device` under NCCL, a CPU tensor under gloo; `x` itself at world 1."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    dev = "cpu" if dist.get_backend() == "gloo" else device
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(units_per_rank, world, seconds_max):
    """Whole-job throughput of `world` independent replicas: every rank processes the same
    units, and the job takes as long as its slowest rank."""
    return units_per_rank * world / seconds_max


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device, self.rows, self._stop = device, [], threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def sm_count(torch, dev):
    return torch.cuda.get_device_properties(dev).multi_processor_count


def roofline(nodes, seconds, sms, max_mhz, traffic, measured=None):
    """INT32-issue roofline of the search kernel: algorithmic lane-ops per second against
    the measured integer issue rate (nqb_measure_int32_peak), the nominal one beside it."""
    achieved = nodes / seconds * INT_OPS_PER_NODE / 1e12
    nominal = sms * 4 * 32 * max_mhz * 1e6 / 1e12
    out = {"bound": "int32-issue", "achieved": round(achieved, 3), "unit": "Tlane-op/s", "traffic": traffic,
           "ops_per_node": INT_OPS_PER_NODE, "peak_nominal": round(nominal, 3),
           "frac_of_nominal": round(achieved / nominal, 4)}
    if measured:
        best, kinds = measured
        out.update(peak=round(best / 1e12, 3), frac=round(achieved / (best / 1e12), 4),
                   peak_source="measured: nqb_measure_int32_peak, best of LOP3 / add / IMAD / LOP3+IMAD chains "
                               "on every SM (" + ", ".join(f"{k} {v / 1e12:.2f}" for k, v in kinds.items()) + " T/s)")
    else:
        out.update(peak=round(nominal, 3), frac=round(achieved / nominal, 4),
                   peak_source=f"nominal issue peak: {sms} SMs x 4 SMSP x 32 lanes x {max_mhz:.0f} MHz")
    return out


def profile_traffic(kernel, n, d):
    """DRAM bytes per launch recorded from an ncu capture in profiles/ (or None)."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith(f"n{n}d{d} "):
            return int(line.split()[1])
    return None


def cpu_baseline_sample(n, d, target_s, steps=1, offset0=0):
    """Times the reference's host DFS (oracle/_ref) on stride samples of the pool with every
    host core; falls back to the oracle port (single core) when the harness is absent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import nqo
    cores = os.cpu_count() or 1
    results = []
    if nqo.ref_available(n):
        probe = nqo.run_ref(n, "cpu", d, cores, 1 << 18, 0)[0]
        rate = probe["nodes"] / max(probe["seconds"], 1e-3)
        total_est = rate * 0 + probe["nodes"] * probe["states"] / max(probe["sampled"], 1)
        stride = max(1, int(total_est / max(rate * target_s, 1.0)))
        for s in range(steps):
            r = nqo.run_ref(n, "cpu", d, cores, stride, (offset0 + s) % stride)[0]
            results.append(dict(r, stride=stride, offset=(offset0 + s) % stride))
        kind, used = "reference", cores
    else:
        probe = nqo.replay_pool(n, d, 1 << 18, 0)
        t0 = time.perf_counter()
        nqo.replay_pool(n, d, 1 << 18, 1)
        rate = probe["nodes"] / max(time.perf_counter() - t0, 1e-3)
        states = nqo.pool_size(n, d)[0]
        stride = max(1, int(probe["nodes"] * (states / max(probe["sampled"], 1)) / max(rate * target_s, 1.0)))
        for s in range(steps):
            t0 = time.perf_counter()
            r = nqo.replay_pool(n, d, stride, (offset0 + s) % stride)
            results.append(dict(r, seconds=time.perf_counter() - t0, stride=stride, offset=(offset0 + s) % stride,
                                states=states))
        kind, used = "port", 1
    return results, kind, used


def run_nqb(args):
    import torch
    import torch.distributed as dist
    rank, world, local = rank_env()
    dev = local
    torch.cuda.set_device(dev)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", dev))
    nqb = load_pkg()
    n, d = args.n, args.depth
    pool = nqb.generate_pool(n, d)
    states = len(pool)
    stack_depth = n - d - 1
    d_pool = torch.from_numpy(pool.view(np.uint8)).to(f"cuda:{dev}")
    slots = max(args.steps, args.warmup)
    d_out = torch.zeros((slots, 4), dtype=torch.int64, device=f"cuda:{dev}")
    # the batched launch's scratch (control words + steal ring), one zeroed buffer per step
    d_scratch = torch.zeros((slots, nqb.BATCHED_SCRATCH_BYTES), dtype=torch.uint8, device=f"cuda:{dev}")
    stream = torch.cuda.current_stream(dev)
    sptr = stream.cuda_stream
    form = {"plain": nqb.FORM_PLAIN, "batched": nqb.FORM_BATCHED}[args.form]

    # autotuned launch: every form and block size timed on a 1/64 stride sample of the pool
    # (depths d-1..d+1 are tuned too: the pick over all of them is run as a full count in extras)
    tuning, blocks = None, {nqb.FORM_PLAIN: args.block, nqb.FORM_BATCHED: args.block}
    if not args.block and not args.no_tune:
        tuning = nqb.tune_count(n, [x for x in (d - 1, d, d + 1) if 1 <= x < n], sample_div=64, device=dev)
        for f in blocks:
            blocks[f] = min((t for t in tuning["tried"] if t["form"] == f and t["depth"] == d),
                            key=lambda t: t["ms"])["block_size"]

    def launch(f, out_row, scratch):
        if f == nqb.FORM_PLAIN:
            nqb.plain_launch(d_pool.data_ptr(), states, out_row.data_ptr(), block_size=blocks[f],
                             stack_depth=stack_depth, stream=sptr)
        else:
            nqb.batched_launch_ex(d_pool.data_ptr(), states, scratch.data_ptr(), scratch.numel(),
                                  out_row.data_ptr(), block_size=blocks[f], stack_depth=stack_depth, stream=sptr)

    def step(i):
        launch(form, d_out[i], d_scratch[i])

    # warm-up (untimed), also the correctness check
    d_out.zero_()
    d_scratch.zero_()
    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize(dev)
    w = d_out.cpu().numpy().astype(np.uint64)
    count, nodes = int(w[0, 0]), int(w[0, 1])
    assert all(int(w[i, 3]) == 0 for i in range(args.warmup)), "device error flag set"
    assert all(int(w[i, 0]) == count and int(w[i, 1]) == nodes for i in range(args.warmup))
    if n in KAT:
        assert count == KAT[n], (count, KAT[n])
    # the roofline's denominator, measured on this GPU before the timed region
    int32_peak = nqb.measure_int32_peak(dev)

    # timed region: K full counts, pool resident in HBM (630 MB > L2 at n=21 d=7)
    d_out.zero_()
    d_scratch.zero_()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(dev) as clk:
        ev0.record(stream)
        for i in range(args.steps):
            step(i)
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    ms = ev0.elapsed_time(ev1)
    res = d_out.cpu().numpy().astype(np.uint64)
    assert all(int(res[i, 0]) == count and int(res[i, 1]) == nodes for i in range(args.steps))
    ms = max_over_ranks(ms, world, f"cuda:{dev}")
    ms_step = ms / args.steps
    value = replica_rate(nodes, world, ms_step / 1e3)

    # the other form on the same resident pool, K steps, for the plain-vs-batched comparison
    forms = {args.form: {"ms": round(ms_step, 3), "nodes_per_s": round(nodes / (ms_step / 1e3), 1),
                         "steps": args.steps}}
    if not args.skip_other_form:
        other = "plain" if args.form == "batched" else "batched"
        d_out.zero_()
        d_scratch.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(args.steps):
            launch({"plain": nqb.FORM_PLAIN, "batched": nqb.FORM_BATCHED}[other], d_out[i], d_scratch[i])
        e1.record(stream)
        torch.cuda.synchronize(dev)
        o = d_out.cpu().numpy().astype(np.uint64)
        assert all(int(o[i, 0]) == count and int(o[i, 1]) == nodes and int(o[i, 3]) == 0 for i in range(args.steps))
        oms = e0.elapsed_time(e1) / args.steps
        forms[other] = {"ms": round(oms, 3), "nodes_per_s": round(nodes / (oms / 1e3), 1), "steps": args.steps}
        if "plain" in forms and "batched" in forms:
            forms["batched_over_plain"] = round(forms["plain"]["ms"] / forms["batched"]["ms"], 3)
    # warp execution efficiency of each form's search loop, from the instrumented kernels
    # (one extra count each, untimed): lane-steps that placed a queen / lane-step slots
    if not args.skip_lane_stats:
        for fname in ([args.form] if args.skip_other_form else ["batched", "plain"]):
            f = {"plain": nqb.FORM_PLAIN, "batched": nqb.FORM_BATCHED}[fname]
            c, st = nqb.count_ex(n, d, device=dev, form=f, block_size=blocks[f], count_lane_steps=True)
            assert c == count and st["nodes"] == nodes
            forms.setdefault(fname, {})
            forms[fname]["lane_efficiency"] = round(st["lane_efficiency"], 4)
            forms[fname]["placed_lane_steps"] = st["placed_lane_steps"]
            forms[fname]["lane_step_slots"] = st["lane_step_slots"]
            forms[fname]["instrumented_kernel_ms"] = round(st["kernel_ms"], 3)

    # e2e: the public C ABI call with host buffers, every step
    e2e = None
    if not args.skip_e2e:
        nqb.count_ex(n, d, device=dev, form=form, block_size=blocks[form])  # warm-up of the call path
        if world > 1:
            dist.barrier()
        walls, gen, h2d, ker, lib_wall = [], [], [], [], []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            c, st = nqb.count_ex(n, d, device=dev, form=form, block_size=blocks[form])
            walls.append(time.perf_counter() - t0)
            assert c == count
            gen.append(st["gen_ms"]), h2d.append(st["h2d_ms"]), ker.append(st["kernel_ms"])
            lib_wall.append(st["wall_ms"])
        wall = max_over_ranks(max(walls), world, f"cuda:{dev}")
        mean_wall = max_over_ranks(sum(walls) / len(walls), world, f"cuda:{dev}")
        # host->device: the row-0 seed states; device->host: 8 bytes of scan totals per pool
        # level, then the 32-byte result
        e2e = {"value": replica_rate(nodes, world, mean_wall), "unit": "nodes/s",
               "h2d_bytes_per_step": 16 * ((n + 1) // 2), "d2h_bytes_per_step": 8 * d + 32,
               "wall_ms_per_step": round(1e3 * mean_wall, 3), "max_wall_ms": round(1e3 * wall, 3),
               "gen_ms": round(float(np.mean(gen)), 3), "h2d_ms": round(float(np.mean(h2d)), 3),
               "kernel_ms": round(float(np.mean(ker)), 3), "api": "nqb_count_ex",
               "wall_ms_steps": [round(1e3 * w, 3) for w in walls],
               "library_wall_ms_steps": [round(w, 3) for w in lib_wall]}
        t0 = time.perf_counter()
        c, st = nqb.count_ex(n, d, device=dev, form=form, block_size=blocks[form], host_pool=True)
        hw = time.perf_counter() - t0
        assert c == count
        e2e["host_pool"] = {"wall_ms": round(1e3 * hw, 3), "gen_ms": round(st["gen_ms"], 3),
                            "h2d_ms": round(st["h2d_ms"], 3), "h2d_bytes": states * 16,
                            "nodes_per_s": round(nodes / hw, 1)}

    extras = None
    if rank == 0 and world == 1 and not args.skip_extras:
        extras = run_extras(nqb, dev, args)
        if tuning:  # the autotuner's own pick (depth, form, block) as a full count
            t0 = time.perf_counter()
            c, st = nqb.count_ex(n, tuning["depth"], device=dev, form=tuning["form"], block_size=tuning["block_size"])
            wall = time.perf_counter() - t0
            extras["autotuned_count"] = {
                "picked": {k: tuning[k] for k in ("depth", "form", "block_size", "split_factor")},
                "count": c, "count_ok": c == count, "wall_ms": round(1e3 * wall, 3), "kernel_ms": round(st["kernel_ms"], 3),
                "over_headline_e2e": round(e2e["wall_ms_per_step"] / (1e3 * wall), 3) if e2e else None}

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        rs, kind, cores = cpu_baseline_sample(n, d, args.cpu_seconds)
        r = rs[0]
        cpu = {"value": r["nodes"] / r["seconds"], "unit": "nodes/s", "cores": cores, "kind": kind,
               "sample": f"every {r['stride']}th state of the n={n} d={d} pool ({r['sampled']} of {r['states']} "
                         f"states, {r['nodes']} nodes, {r['seconds']:.2f} s)"}
        # the same sample through the library: bit-exact check of the baseline's count
        samp = pool[r["offset"]::r["stride"]]
        got, stc = nqb.solve_states(samp, device=dev)
        cpu["sample_count_match"] = bool(got == r["count"] and stc["nodes"] == r["nodes"])

    if rank == 0:
        sms = sm_count(torch, dev)
        ck = clk.summary()
        max_mhz = ck["sm_max_mhz"] or 1965.0
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": "nodes/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_step, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic (the full depth-7 pool of the N=21 board)",
            "config": {"workload": f"full count N={n}, pregen depth {d}", "n": n, "depth": d, "form": args.form,
                       "states": states, "nodes": nodes, "count": count, "block": blocks[form] or 128,
                       "other_form_block": blocks[1 - form] or 128, "tuning": tuning,
                       "parallelism": f"replicas{world}" if world > 1 else "single",
                       "schedule": "FIFO with work stealing: the learned scheduler leaves a queue of more than "
                                   "64 items per resident lane unchanged (39.4M items at N=21 d=7), so the "
                                   "headline is the batched form as given; extras.ablation measures the "
                                   "learned schedule where it acts",
                       "l2": f"inputs larger than L2 (pool {states * 16 / 1e6:.0f} MB)"},
            "forms": forms,
            "e2e": e2e,
            "roofline": roofline(nodes, ms_step / 1e3, sms, max_mhz,
                                 profile_traffic(f"{args.form}_search_kernel", n, d), int32_peak),
            "cpu_baseline": cpu,
            "clocks": ck,
            "gpu_launches": args.steps * (1 + (states - 1) // (1 << 30)),
            "extras": extras,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def _spearman(a, b):
    rank = lambda v: np.argsort(np.argsort(v, kind="stable"), kind="stable").astype(np.float64)
    return float(np.corrcoef(rank(a), rank(b))[0, 1])


def run_extras(nqb, dev, args):
    """The learned model and the other workloads of the project, beside the headline (not timed
    as the bench value): the cost model trained on 1M seeded N=18 prefixes (depth 4..8) with
    node counts recorded by the solver, its accuracy on the N=19 depth-5 pool it never saw, and
    an ablation of the split-and-order schedule it drives against the same pipeline driven by an
    untrained network and by two model-free costs, on the N=19 depth-4 and N=17 depth-3 counts
    and on the 65,536 uneven partial boards (autotuned CUDA-graph plans)."""
    out = {}
    t0 = time.perf_counter()
    boards = nqb.sample_boards(nqb.MODEL_SEED, args.model_samples, 18, 18, 4, 8)
    nodes, _ = nqb.record_nodes(boards, device=dev)
    t = np.log2(1.0 + nodes.astype(np.float64)).astype(np.float32)
    ntr = int(0.9 * len(boards))
    t1 = time.perf_counter()
    model = nqb.Model(device=dev, seed=1)
    losses = model.train(boards[:ntr], t[:ntr], epochs=8, batch=4096, lr=2e-3)
    t2 = time.perf_counter()
    pred = model.predict(boards[ntr:])
    out["model"] = {"samples": len(boards), "train": ntr, "train_set": "n=18, depth 4..8 (seeded sampler)",
                    "label_nodes": int(nodes.sum()), "label_s": round(t1 - t0, 2), "train_s": round(t2 - t1, 2),
                    "epoch_loss": [round(float(x), 4) for x in losses],
                    "val_rmse_log2": round(float(np.sqrt(np.mean((pred - t[ntr:]) ** 2))), 4),
                    "val_std_log2": round(float(np.std(t[ntr:])), 4),
                    "val_spearman": round(_spearman(pred, t[ntr:]), 4)}
    # transfer to a board size the network never saw: the N=19 depth-5 pool
    pool = nqb.generate_pool(19, 5)
    pn, _ = nqb.record_nodes(pool, device=dev)
    pt = np.log2(1.0 + pn.astype(np.float64))
    pp = model.predict(pool).astype(np.float64)
    out["model"]["n19_d5_pool"] = {"items": len(pool), "rmse_log2": round(float(np.sqrt(np.mean((pp - pt) ** 2))), 4),
                                   "std_log2": round(float(np.std(pt)), 4), "spearman": round(_spearman(pp, pt), 4)}
    # the same network trained on mixed board sizes (n 16..20, depth 4..8), reported beside it
    mb = nqb.sample_boards(nqb.MODEL_SEED, args.model_samples, 16, 20, 4, 8)
    mn, _ = nqb.record_nodes(mb, device=dev)
    mt = np.log2(1.0 + mn.astype(np.float64)).astype(np.float32)
    mixed = nqb.Model(device=dev, seed=1)
    mixed.train(mb[:ntr], mt[:ntr], epochs=8, batch=4096, lr=2e-3)
    mp = mixed.predict(mb[ntr:])
    qp = mixed.predict(pool).astype(np.float64)
    out["model_mixed_n"] = {"train_set": "n=16..20, depth 4..8 (seeded sampler)", "samples": len(mb),
                            "val_rmse_log2": round(float(np.sqrt(np.mean((mp - mt[ntr:]) ** 2))), 4),
                            "val_std_log2": round(float(np.std(mt[ntr:])), 4),
                            "val_spearman": round(_spearman(mp, mt[ntr:]), 4),
                            "n19_d5_pool": {"rmse_log2": round(float(np.sqrt(np.mean((qp - pt) ** 2))), 4),
                                            "std_log2": round(float(np.std(pt)), 4),
                                            "spearman": round(_spearman(qp, pt), 4)}}
    untrained = nqb.Model(device=dev, seed=1)
    arms = {"fifo": {}, "untrained_net": {"model": untrained}, "free_x_rows": {"sched_cost": 1},
            "lookahead_cells": {"sched_cost": 2}, "trained_net": {"model": model},
            "trained_mixed_n": {"model": mixed}}

    # the ablation on coarse full counts: kernel + scheduling time of each arm (second of two runs)
    abl = {}
    for n, d in ((19, 4), (17, 3)):
        row = {}
        for name, kw in arms.items():
            for _ in range(2):
                c, st = nqb.count_ex(n, d, device=dev, form=nqb.FORM_BATCHED, **kw)
            assert c == KAT[n]
            row[name] = {"kernel_ms": round(st["kernel_ms"], 3), "sched_ms": round(st["sched_ms"], 3),
                         "items": st["items"]}
        abl[f"n{n}_d{d}"] = row

    # uneven partial boards (65,536, n 16..20, depth 3..7): an autotuned plan per arm
    cb = nqb.sample_boards(nqb.BATCH_SEED, 65536, 16, 20, 3, 7)
    fifo, st_f = nqb.solve_batch(cb, device=dev, form=nqb.FORM_BATCHED)
    plain_ub, st_p0 = nqb.solve_batch(cb, device=dev, form=nqb.FORM_PLAIN)
    assert np.array_equal(plain_ub, fifo)
    row = {}
    for name, kw in arms.items():
        tc = time.perf_counter()
        plan = nqb.BatchPlan(cb, device=dev, autotune=True, **kw)
        tc = time.perf_counter() - tc
        runs = []
        for _ in range(3):
            got, st_p = plan.run()
            assert np.array_equal(got, fifo)
            runs.append(st_p["kernel_ms"])
        row[name] = {"plan_create_s": round(tc, 3), "run_ms": [round(x, 2) for x in runs], "plan": plan.config()}
        plan.close()
    abl["uneven_boards"] = row
    out["ablation"] = abl
    best = min(row["trained_net"]["run_ms"])
    out["uneven_boards"] = {
        "boards": len(cb), "nodes": st_f["nodes"], "sum_counts": int(fifo.sum()), "bit_exact": True,
        "plain_ms": round(st_p0["kernel_ms"], 2), "batched_fifo_ms": round(st_f["kernel_ms"], 2),
        "learned_plan_ms": best, "learned_over_fifo": round(st_f["kernel_ms"] / best, 3),
        "plan_create_s": row["trained_net"]["plan_create_s"],
        "e2e_over_fifo": round(st_f["kernel_ms"] / (1e3 * row["trained_net"]["plan_create_s"] + best), 3)}

    # N=19 full counts: plain, batched FIFO, batched + learned
    n19 = {}
    for d in (4, 7):
        c0, s0 = nqb.count_ex(19, d, device=dev, form=nqb.FORM_PLAIN)
        c1, s1 = nqb.count_ex(19, d, device=dev, form=nqb.FORM_BATCHED)
        c2, s2 = nqb.count_ex(19, d, device=dev, form=nqb.FORM_BATCHED, model=model)
        assert c0 == c1 == c2 == KAT[19] and s0["nodes"] == s1["nodes"] == s2["nodes"]
        n19[f"d{d}"] = {"plain_ms": round(s0["kernel_ms"], 2), "batched_ms": round(s1["kernel_ms"], 2),
                        "learned_ms": round(s2["kernel_ms"], 2), "learned_sched_ms": round(s2["sched_ms"], 2),
                        "learned_items": s2["items"], "learned_over_plain": round(s0["kernel_ms"] / s2["kernel_ms"], 3)}
    out["n19"] = n19
    untrained.close()
    mixed.close()
    model.close()
    return out


def run_reference(args):
    rank, world, local = rank_env()
    if rank != 0:
        return
    n, d = args.n, args.depth
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import nqo
    step_s = args.ref_step_seconds
    rs, kind, cores = cpu_baseline_sample(n, d, step_s, steps=args.warmup + args.steps)
    timed = rs[args.warmup:]
    nodes = sum(r["nodes"] for r in timed)
    secs = sum(r["seconds"] for r in timed)
    value = nodes / secs
    sample = (f"per step every {timed[0]['stride']}th state of the n={n} d={d} pool (offsets "
              f"{[r['offset'] for r in timed]}), {nodes} nodes in {secs:.2f} s")
    line = {"metric": METRIC, "impl": "reference", "value": round(value, 1), "unit": "nodes/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * secs / len(timed), 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (stride samples of the depth-7 pool of the N=21 board)",
            "config": {"workload": f"full count N={n}, pregen depth {d}", "n": n, "depth": d,
                       "form": "reference host DFS (locked_advance_nq_state)"},
            "cpu_baseline": {"value": round(value, 1), "unit": "nodes/s", "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": round(value, 1), "unit": "nodes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    rn, rd = args.ref_cuda_n, args.ref_cuda_d
    if args.ref_cuda and nqo.ref_available(rn):
        line["reference_cuda"] = reference_cuda(nqo, rn, rd)
    print(json.dumps(line), flush=True)


def reference_cuda(nqo, n, d):
    """The reference CUDA build (kern_doitall_v2_regld via gpu_solver_driver) on this GPU."""
    import re
    t0 = time.perf_counter()
    p = subprocess.run([nqo.ref_harness_path(n), "gpu", str(d), "1"], capture_output=True, text=True, timeout=3600)
    wall = time.perf_counter() - t0
    if p.returncode != 0:
        return {"unavailable": f"reference CUDA run exited {p.returncode}"}
    js = [json.loads(l[9:]) for l in p.stdout.splitlines() if l.startswith("NQO_JSON ")]
    km = [float(x) for x in re.findall(r"Time taken: ([0-9.]+)ms", p.stdout)]
    r = js[-1] if js else {}
    out = {"workload": f"full count N={n}, pregen depth {d}", "count": r.get("count"),
           "count_ok": r.get("count") == KAT.get(n), "kernel_ms": km[-1] if km else None,
           "driver_ms": round(1e3 * r.get("driver_seconds", 0), 3), "gen_ms": round(1e3 * r.get("gen_seconds", 0), 3),
           "process_wall_s": round(wall, 3)}
    if (n, d) in NODES and out["kernel_ms"]:
        out["nodes_per_s"] = round(NODES[(n, d)] / (out["kernel_ms"] / 1e3), 1)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="nqb", choices=["nqb", "reference"])
    ap.add_argument("--n", type=int, default=21)
    ap.add_argument("--depth", type=int, default=7)
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--form", default="batched", choices=["batched", "plain"])
    ap.add_argument("--skip-other-form", action="store_true")
    ap.add_argument("--skip-extras", action="store_true")
    ap.add_argument("--model-samples", type=int, default=1000000)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-step-seconds", type=float, default=8.0)
    ap.add_argument("--ref-cuda", type=int, default=1)
    ap.add_argument("--ref-cuda-n", type=int, default=21)
    ap.add_argument("--ref-cuda-d", type=int, default=7)
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-lane-stats", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="skip the launch autotuner (default block sizes)")
    args = ap.parse_args()
    if args.warmup < 1:
        args.warmup = 1
    if args.impl == "reference":
        run_reference(args)
    else:
        run_nqb(args)


if __name__ == "__main__":
    main()
