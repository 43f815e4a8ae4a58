"""Regenerates tests/golden/ref_vectors.json from the reference itself.

Run where the reference's sources are (it reads them and runs oracle/_ref, the
reference's own code built by `make -C oracle ref REF_DIR=<reference checkout>`):

    python tests/golden/make_golden.py --reference <reference checkout> [--quick]

(`--reference` may be left out when NQB_REFERENCE_DIR names the checkout.)

Captured:
  kat_counts       the known-answer table of check_if_known_result (test.cu:17-24)
  pool_file_sizes  (n, lock row, weighted pool size) from the pool file names of
                   pre_gen_state_files (test.cu:87-105)
  pools            ref_harness `pool`: size, weighted size, FNV-1a hash of every
                   state's (curr_row, queen columns) in generation order
  replays          ref_harness `replay`: the reference kernel loop replayed on the host
                   over the pool (or a stride sample of it): weighted count, nodes, unit
"""
import argparse
import json
import os
import re
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_SRC = None  # the reference checkout: --reference, else NQB_REFERENCE_DIR
HARNESS = os.path.join(ROOT, "oracle", "_ref", "N{n}", "ref_harness")

POOLS = [(n, d) for n in range(8, 15) for d in range(1, n)] + [
    (15, 4), (16, 5), (17, 5), (17, 8), (18, 4), (18, 5), (18, 6), (18, 7), (18, 8), (19, 7), (20, 7),
    (21, 5), (21, 6), (21, 7), (22, 6), (22, 7)]
REPLAYS = ([(n, d, 1, 0) for n in range(8, 13) for d in range(1, n)]
           + [(13, 3, 1, 0), (13, 5, 1, 0), (14, 4, 1, 0), (15, 4, 1, 0), (16, 5, 1, 0),
              (17, 5, 1, 0), (18, 6, 64, 0), (19, 7, 512, 3), (20, 7, 4096, 5), (21, 7, 16384, 0),
              (22, 7, 131072, 7)])
QUICK_SKIP = {(16, 5), (17, 5), (18, 6), (19, 7), (20, 7), (21, 7), (22, 7)}


def run(n, *args):
    out = subprocess.run([HARNESS.format(n=n)] + [str(a) for a in args], capture_output=True, text=True,
                         check=True).stdout
    return [json.loads(l[len("NQO_JSON "):]) for l in out.splitlines() if l.startswith("NQO_JSON ")][-1]


def read_test_tables():
    src = open(os.path.join(REF_SRC, "test.cu"), encoding="utf-8-sig").read()
    m = re.search(r"results\[\]\s*=\s*\{([^}]*)\}", src)
    kat = [int(x.strip().rstrip("ULL").rstrip("U")) for x in m.group(1).split(",") if x.strip()]
    files = [{"n": int(a), "weighted": int(b), "d": int(c)}
             for a, b, c in re.findall(r"n(\d+)_(\d+)_lk(\d+)_valid\.nqsb", src)]
    return {str(i + 1): v for i, v in enumerate(kat)}, files


def main():
    global REF_SRC
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", default=os.environ.get("NQB_REFERENCE_DIR"),
                    help="the reference checkout (default: $NQB_REFERENCE_DIR)")
    ap.add_argument("--quick", action="store_true", help="keep the largest replays from the existing file")
    args = ap.parse_args()
    if not args.reference or not os.path.isfile(os.path.join(args.reference, "test.cu")):
        ap.error("--reference (or NQB_REFERENCE_DIR) must name the reference checkout")
    REF_SRC, quick = args.reference, args.quick
    kat, files = read_test_tables()
    with ThreadPoolExecutor(max_workers=os.cpu_count()) as ex:
        pools = list(ex.map(lambda nd: run(nd[0], "pool", nd[1]), POOLS))
        reps = [r for r in REPLAYS if not (quick and (r[0], r[1]) in QUICK_SKIP)]
        replays = list(ex.map(lambda r: dict(run(r[0], "replay", r[1], r[2], r[3]), stride=r[2], offset=r[3]),
                              reps))
    out = {"source": "fillpant/GPU-N-Queens test.cu and oracle/_ref (the reference's own code)",
           "kat_counts": kat, "pool_file_sizes": files, "pools": pools, "replays": replays}
    path = os.path.join(HERE, "ref_vectors.json")
    if quick and os.path.exists(path):
        old = json.load(open(path))
        keep = [r for r in old.get("replays", []) if (r["n"], r["d"]) in QUICK_SKIP]
        out["replays"] = replays + keep
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {path}: {len(pools)} pools, {len(out['replays'])} replays")


if __name__ == "__main__":
    main()
