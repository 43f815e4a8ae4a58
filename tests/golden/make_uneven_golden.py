"""Regenerates tests/golden/uneven_boards.json: the reference's own counts for a stratified
sample of the uneven partial-board batch (65,536 boards, n uniform in 16..20, depth uniform
in 3..7, seed 0x4E51554545534231; the library's nqb_sample_boards).

Each sampled board is rebuilt by the reference's init_nq_state + place_queen_at from its
queen columns and streamed with locked_advance_nq_state(depth, n-1) (n_queens.cu:423-445)
by `oracle/_ref/N<n>/ref_harness boards`, with no mirror weight: the completions and the
placements below the board's last row.  Run where `make -C oracle ref REF_DIR=...` has
built the harnesses:

    python tests/golden/make_uneven_golden.py [--sizes nodes.npy]

Selection: every (n, depth) cell contributes its largest board and 7 more drawn with a
fixed seed from the rest of the cell.  "Largest" needs every board's node count, which
only a GPU run gives in reasonable time: --sizes names a .npy of the 65,536 per-board
node counts (nqb.record_nodes on the batch).  Without it the indices already in the
fixture are kept and only the reference's values are regenerated.
"""
import argparse
import json
import os
import subprocess
import tempfile
from concurrent.futures import ThreadPoolExecutor

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "N{n}", "ref_harness")
OUT = os.path.join(HERE, "uneven_boards.json")
SEED, COUNT, N_MIN, N_MAX, D_MIN, D_MAX = 0x4E51554545534231, 65536, 16, 20, 3, 7
PER_CELL = 8
M64 = (1 << 64) - 1


class SplitMix64:
    """The generator of nqb_sample_boards (pool.cpp): splitmix64 and a 32x32-bit range map."""

    def __init__(self, seed):
        self.s = seed & M64

    def next(self):
        self.s = (self.s + 0x9E3779B97F4A7C15) & M64
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        return z ^ (z >> 31)

    def below(self, k):
        return ((self.next() >> 32) * k) >> 32


def sample_boards(seed, count, n_min, n_max, d_min, d_max):
    """(n, depth, queen columns, (cols, ldiag, rdiag)) of every board, as nqb_sample_boards
    draws them: rows in order, each column uniform over the free ones, restart on a dead end."""
    rng = SplitMix64(seed)
    out = []
    for _ in range(count):
        n = n_min + rng.below(n_max - n_min + 1)
        d = d_min + rng.below(d_max - d_min + 1)
        mask = (1 << n) - 1
        while True:
            cols = ld = rd = 0
            q = []
            for _r in range(d):
                f = mask & ~(cols | ld | rd)
                if not f:
                    break
                for _k in range(rng.below(bin(f).count("1"))):
                    f &= f - 1
                b = f & -f
                q.append(b.bit_length() - 1)
                cols |= b
                ld = ((ld | b) << 1) & 0xFFFFFFFF
                rd = (rd | b) >> 1
            if len(q) == d:
                break
        out.append((n, d, q, (cols, ld, rd)))
    return out


def select(boards, sizes):
    rng = np.random.default_rng(1)
    picked = []
    for n in range(N_MIN, N_MAX + 1):
        for d in range(D_MIN, D_MAX + 1):
            cell = [i for i, b in enumerate(boards) if b[0] == n and b[1] == d]
            big = max(cell, key=lambda i: int(sizes[i]))
            rest = [i for i in cell if i != big]
            picked += [big] + sorted(rng.choice(rest, size=min(PER_CELL - 1, len(rest)), replace=False).tolist())
    return sorted(picked)


def reference_values(boards, picked):
    by_n = {}
    for i in picked:
        by_n.setdefault(boards[i][0], []).append(i)

    def run(n):
        with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
            for i in by_n[n]:
                f.write(" ".join(str(x) for x in [boards[i][1]] + boards[i][2]) + "\n")
            path = f.name
        try:
            out = subprocess.run([HARNESS.format(n=n), "boards", path, str(os.cpu_count() or 1)],
                                 capture_output=True, text=True, check=True).stdout
        finally:
            os.unlink(path)
        js = [json.loads(l[len("NQO_JSON "):]) for l in out.splitlines() if l.startswith("NQO_JSON ")][-1]
        return {i: (c, m) for i, c, m in zip(by_n[n], js["count"], js["nodes"])}

    vals = {}
    for n in sorted(by_n):  # one board size at a time, each with every host core
        vals.update(run(n))
    return vals


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--sizes", help=".npy of the batch's per-board node counts, to select the sample anew")
    args = ap.parse_args()
    boards = sample_boards(SEED, COUNT, N_MIN, N_MAX, D_MIN, D_MAX)
    if args.sizes:
        picked = select(boards, np.load(args.sizes))
        how = "per (n, depth) cell: the largest board by node count and 7 more drawn with seed 1"
    else:
        old = json.load(open(OUT))
        picked, how = [b["index"] for b in old["boards"]], old["selection"]
    vals = reference_values(boards, picked)
    out = {"source": "oracle/_ref ref_harness boards: the reference's locked_advance_nq_state per board",
           "seed": SEED, "count": COUNT, "n": [N_MIN, N_MAX], "depth": [D_MIN, D_MAX], "selection": how,
           "boards": [{"index": i, "n": boards[i][0], "d": boards[i][1], "cols": boards[i][2],
                       "masks": list(boards[i][3]), "count": vals[i][0], "nodes": vals[i][1]} for i in picked]}
    with open(OUT, "w") as f:
        json.dump(out, f, indent=0)
    print(f"wrote {OUT}: {len(picked)} boards, {sum(v[1] for v in vals.values())} nodes")


if __name__ == "__main__":
    main()
