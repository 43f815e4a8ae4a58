"""The nqb_solver command line against the reference's NQ_solver.

CPU: every state file the reference CLI wrote for the fixtures (row-lock and count-target
pools, shuffled with and without a seed, split into chunks) is written byte for byte the
same from the same arguments, and the argument and error paths exit as the reference's do.
GPU: solving files and count-target pools prints the known counts."""
import json
import os
import re
import subprocess

import pytest

from conftest import GOLDEN_DIR, PKG_DIR

GOLD = json.load(open(os.path.join(GOLDEN_DIR, "nqsf_vectors.json")))
KAT = {int(k): v for k, v in json.load(open(os.path.join(GOLDEN_DIR, "ref_vectors.json")))["kat_counts"].items()}
NQSF_DIR = os.path.join(GOLDEN_DIR, "nqsf")
CLI = os.path.join(PKG_DIR, "nqb_solver")


def run(*args, cwd=None, timeout=600):
    if not os.access(CLI, os.X_OK):
        pytest.fail(f"{CLI} is not built: run `make -C {PKG_DIR}`")
    return subprocess.run([CLI] + [str(a) for a in args], capture_output=True, text=True, cwd=cwd, timeout=timeout)


@pytest.mark.parametrize("f", [f for f in GOLD["files"] if "args" in f], ids=lambda f: f["name"])
def test_generated_files_match_reference_cli(f, tmp_path):
    out = tmp_path / "out.nqsf"
    p = run("-n", f["n"], *[a.format(out=out) for a in f["args"]])
    assert p.returncode == 0, p.stderr
    assert out.read_bytes() == open(os.path.join(NQSF_DIR, f["name"]), "rb").read()


@pytest.mark.parametrize("d", GOLD["dirs"], ids=lambda d: d["name"])
def test_chunk_files_match_reference_cli(d, tmp_path):
    p = run("-n", d["n"], *[a.format(out=tmp_path) for a in d["args"]])
    assert p.returncode == 0, p.stderr
    assert sorted(os.listdir(tmp_path)) == sorted(c["name"] for c in d["chunks"])
    for c in d["chunks"]:
        assert (tmp_path / c["name"]).read_bytes() == open(os.path.join(NQSF_DIR, d["name"], c["name"]), "rb").read()


def test_count_target_messages(tmp_path):
    """`-g` prints one line per lock row tried, as the reference does."""
    row = next(r for r in GOLD["targets"]["10"] if r.get("lock") == 4)
    p = run("-n", 10, "-g", row["h"], "-w", tmp_path / "t.nqsf")
    assert p.returncode == 0
    tried = [int(x) for x in re.findall(r"Lock at row \d+\.\.\. (\d+) states generated", p.stdout)]
    assert tried == row["tried"]


@pytest.mark.parametrize("args,message", [
    (["-R", "3", "-g", "100", "-w", "x"], "must not be combined"),
    (["-R", "3"], "no output file supplied"),
    (["-g", "0", "-w", "x"], "Cannot generate"),
    (["-R", "-2", "-w", "x"], "Cannot lock at row"),
    (["-R", "8", "-w", "x"], "Cannot lock at row"),         # row >= N
    (["-s", "0", "-R", "3", "-w", "x"], "Count value"),
    (["-t", "abc"], "Cannot try with"),
    (["-r", "-1", "-R", "3", "-w", "x"], "Seed"),
    (["-d", "0,,1", "-R", "3", "-w", "x"], "Failed to parse GPU list"),
    (["-d", "", "-R", "3", "-w", "x"], "Failed to parse GPU list"),
    (["-n", "40"], "Board size"),
    (["-f", "fast"], "Unknown form"),
    (["-g", "5", "-w", "x"], "status 1"),                   # lock row 0 (n_queens.cu:139)
    (["-g", "10", "-w", "x"], "status 5"),                  # no row within the limit (:196)
    (["-l", "missing.nqsf"], "Failed to read states"),
])
def test_argument_errors(args, message, tmp_path):
    p = run("-n", 8, *args, cwd=tmp_path)
    assert p.returncode == 1 and message in p.stderr, p.stderr


def test_more_chunks_than_states_fails_like_reference(tmp_path):
    # 21 states over 30 chunks: the first 21 files get one state, the 22nd none, and the
    # reference writer refuses an empty chunk
    p = run("-n", 8, "-R", "1", "-s", "30", "-w", tmp_path)
    assert p.returncode == 1 and "Failed to write chunk" in p.stderr
    assert len(os.listdir(tmp_path)) == 21


def test_help_and_unknown_options(tmp_path):
    p = run("-h")
    assert p.returncode == 0 and "--gen-rowlock" in p.stdout and "--load-states" in p.stdout
    p = run("-n", 8, "-x", "-R", "3", "-w", tmp_path / "a.nqsf")  # unknown options are reported, then ignored
    assert p.returncode == 0 and "Unsupported argument '-x'" in p.stderr
    p = run("--board=8", "--gen-rowlock", "3", "--write-states=" + str(tmp_path / "b.nqsf"))
    assert p.returncode == 0
    assert (tmp_path / "b.nqsf").read_bytes() == open(os.path.join(NQSF_DIR, "R_n8_l3.nqsf"), "rb").read()


def test_load_rejects_other_board_size():
    p = run("-n", 9, "-l", os.path.join(NQSF_DIR, "R_n8_l3.nqsf"))
    assert p.returncode == 1 and "Failed to read states" in p.stderr


def solution(p):
    m = re.search(r"solution_count\((\d+)\) = (\d+) \(([\d,]+)\)", p.stdout)
    assert p.returncode == 0 and m, p.stdout + p.stderr
    assert m.group(3).replace(",", "") == m.group(2)
    return int(m.group(1)), int(m.group(2))


@pytest.mark.gpu
@pytest.mark.parametrize("f", GOLD["files"], ids=lambda f: f["name"])
def test_solve_reference_files(f):
    """Every whole-pool fixture counts the board's solutions (the mixed-row files are not
    whole pools and are covered by the library's mixed-board tests)."""
    if "mix" in f:
        pytest.skip("not a whole pool")
    n, c = solution(run("-l", os.path.join(NQSF_DIR, f["name"])))
    assert n == f["n"] and c == KAT[n]


@pytest.mark.gpu
def test_solve_chunks_sum_to_count():
    for d in GOLD["dirs"]:
        total = sum(solution(run("-l", os.path.join(NQSF_DIR, d["name"], c["name"]), "-m"))[1] for c in d["chunks"])
        assert total == KAT[d["n"]]


@pytest.mark.gpu
@pytest.mark.parametrize("args,n", [
    (["-n", 13, "-t", 1000], 13),
    (["-n", 14, "-t", 5000, "-d", "0,0"], 14),          # split across two solver threads
    (["-n", 15, "-t", 100000, "-f", "plain", "-d", "0"], 15),
    (["-n", 16], 16),                                    # the reference's default target (80M)
])
def test_count_target_solve(args, n):
    got_n, c = solution(run(*args))
    assert got_n == n and c == KAT[n]


@pytest.mark.parametrize("lock,states", [(2, 2), (3, 1)])
def test_shuffle_of_tiny_pools_keeps_order(lock, states, tmp_path, nqsf):
    """The reference's shuffle loops over [0, len - 2), which wraps below two states (it
    would run off the buffer); here fewer than three states keep their order, and the file
    equals the unshuffled one."""
    a, b = tmp_path / "m.nqsf", tmp_path / "p.nqsf"
    assert run("-n", 4, "-R", lock, "-m", "-w", a).returncode == 0
    assert run("-n", 4, "-R", lock, "-w", b).returncode == 0
    assert a.read_bytes() == b.read_bytes()
    assert nqsf.read_bytes(a.read_bytes())[4] == states
    assert nqsf.shuffle_perm(states) == list(range(states))
