"""Regenerates tests/golden/nqsf/ and tests/golden/nqsf_vectors.json from the reference itself.

Run in the build container, after `make -C oracle ref cli` (the reference's own CLI and
harness, built from its sources by oracle/Makefile):

    python tests/golden/make_nqsf_golden.py

Captured, all by the reference's own code:
  files     state files written by the reference CLI (NQ_solver -R / -g with -w, -s, -m, -r)
            and by its writer on a mixed-row buffer (ref_harness writemix), with what the
            reference reader makes of each (ref_harness readfile: states, lock, hash)
  targets   the count-target sizing of `NQ_solver -g <how_many>` over a grid of targets:
            the lock row and pool size written, or how the reference failed
"""
import hashlib
import json
import os
import shutil
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref", "N{n}")
OUT_DIR = os.path.join(HERE, "nqsf")

# (name, n, CLI arguments after the output option); `{out}` is the output file or directory
CLI_FILES = [
    ("R_n8_l3", 8, ["-R", "3", "-w", "{out}"]),
    ("R_n9_l1", 9, ["-R", "1", "-w", "{out}"]),
    ("R_n10_l4", 10, ["-R", "4", "-w", "{out}"]),
    ("R_n12_l4", 12, ["-R", "4", "-w", "{out}"]),
    ("g_n9_1000", 9, ["-g", "1000", "-w", "{out}"]),
    ("g_n10_1334", 10, ["-g", "1334", "-w", "{out}"]),
    ("Rm_n9_l4_r7", 9, ["-R", "4", "-m", "-r", "7", "-w", "{out}"]),
    ("Rm_n8_l3_noseed", 8, ["-R", "3", "-m", "-w", "{out}"]),
]
CLI_DIRS = [
    ("Rs_n10_l4_s3", 10, ["-R", "4", "-s", "3", "-w", "{out}"]),
    ("Rs_n11_l3_s5", 11, ["-R", "3", "-s", "5", "-w", "{out}"]),
    ("Rsm_n10_l4_s3_r11", 10, ["-r", "11", "-R", "4", "-m", "-s", "3", "-w", "{out}"]),
]
MIXES = [("mix_n9_3_5", 9, 3, 5), ("mix_n11_4_2", 11, 4, 2)]
TARGET_NS = range(8, 15)
TARGETS = sorted({int(round(10 ** (e / 8))) for e in range(0, 8 * 7 + 1)})


def sha(path):
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def readback(n, path):
    out = subprocess.run([os.path.join(REF.format(n=n), "ref_harness"), "readfile", path], capture_output=True,
                         text=True, check=True).stdout
    return json.loads([l for l in out.splitlines() if l.startswith("NQO_JSON ")][-1][9:])


def cli(n, args, cwd):
    return subprocess.run([os.path.join(REF.format(n=n), "NQ_solver")] + args, capture_output=True, text=True,
                          cwd=cwd, timeout=600)


def main():
    if os.path.isdir(OUT_DIR):
        shutil.rmtree(OUT_DIR)
    os.makedirs(OUT_DIR)
    files, dirs = [], []
    with tempfile.TemporaryDirectory() as tmp:
        for name, n, args in CLI_FILES:
            dst = os.path.join(OUT_DIR, name + ".nqsf")
            p = cli(n, [a.format(out=dst) for a in args], tmp)
            assert p.returncode == 0, p.stdout + p.stderr
            files.append({"name": name + ".nqsf", "n": n, "args": args, "sha256": sha(dst), "ref_read": readback(n, dst)})
        for name, n, args in CLI_DIRS:
            dst = os.path.join(OUT_DIR, name)
            os.makedirs(dst)
            p = cli(n, [a.format(out=dst) for a in args], tmp)
            assert p.returncode == 0, p.stdout + p.stderr
            chunks = []
            for fn in sorted(os.listdir(dst), key=lambda s: int(s.split("_")[1])):
                chunks.append({"name": fn, "sha256": sha(os.path.join(dst, fn)),
                               "ref_read": readback(n, os.path.join(dst, fn))})
            dirs.append({"name": name, "n": n, "args": args, "chunks": chunks})
        for name, n, d1, d2 in MIXES:
            dst = os.path.join(OUT_DIR, name + ".nqsf")
            subprocess.run([os.path.join(REF.format(n=n), "ref_harness"), "writemix", str(d1), str(d2), dst],
                           capture_output=True, check=True)
            files.append({"name": name + ".nqsf", "n": n, "mix": [d1, d2], "sha256": sha(dst),
                          "ref_read": readback(n, dst)})
        targets = {}
        for n in TARGET_NS:
            rows = []
            for h in TARGETS:
                f = os.path.join(tmp, "t.nqsf")
                if os.path.exists(f):
                    os.remove(f)
                p = cli(n, ["-g", str(h), "-w", f], tmp)
                tried = [int(l.split("... ")[1].split()[0]) for l in p.stdout.split("Lock at row ")[1:]
                         if "states generated" in l.split("\n")[0]]
                if p.returncode == 0:
                    b = open(f, "rb").read()
                    rows.append({"h": h, "lock": b[13], "count": int.from_bytes(b[14:22], "little"), "tried": tried})
                elif p.returncode < 0:
                    rows.append({"h": h, "crash": -p.returncode, "tried": tried})
                else:
                    line = "139" if "line 139" in p.stdout + p.stderr else "196" if "line 196" in p.stdout + p.stderr else "?"
                    rows.append({"h": h, "fail_line": line, "tried": tried})
            targets[str(n)] = rows
    json.dump({"files": files, "dirs": dirs, "targets": targets}, open(os.path.join(HERE, "nqsf_vectors.json"), "w"),
              indent=1)
    print(f"{len(files)} files, {len(dirs)} chunk sets, {sum(len(v) for v in targets.values())} targets")


if __name__ == "__main__":
    main()
