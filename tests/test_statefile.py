"""State files (.nqsf), placements and count-target pool sizing, on the CPU.

The oracle (oracle/nqsf.py) is pinned to files the reference's own CLI and writer produced
(tests/golden/nqsf/, made by tests/golden/make_nqsf_golden.py); the library's writer,
reader and sizing are then checked against both, byte for byte."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN_DIR

GOLD = json.load(open(os.path.join(GOLDEN_DIR, "nqsf_vectors.json")))
NQSF_DIR = os.path.join(GOLDEN_DIR, "nqsf")
R_FILES = [f for f in GOLD["files"] if "args" in f and f["args"][0] == "-R" and "-m" not in f["args"]]


def golden_bytes(*parts):
    return open(os.path.join(NQSF_DIR, *parts), "rb").read()


def lock_of(args):
    return int(args[args.index("-R") + 1])


def placements_array(nqb, n, pl):
    """Oracle (row, columns) list -> PLACEMENT_DTYPE array."""
    a = np.zeros(len(pl), dtype=nqb.PLACEMENT_DTYPE)
    a["n"] = n
    a["col"] = 0xFF
    for i, (r, cols) in enumerate(pl):
        a[i]["row"] = r
        a[i]["col"][:r] = cols
    return a


# ---- the oracle against the reference's own files -----------------------------------


@pytest.mark.parametrize("f", R_FILES, ids=lambda f: f["name"])
def test_oracle_writes_reference_rowlock_files(nqsf, f):
    n, lock = f["n"], lock_of(f["args"])
    assert nqsf.write_bytes(n, lock, nqsf.pool_placements(n, lock)) == golden_bytes(f["name"])


@pytest.mark.parametrize("f", GOLD["files"], ids=lambda f: f["name"])
def test_oracle_reads_reference_files(nqsf, f):
    version, flags, n, lock, total, pl = nqsf.read_bytes(golden_bytes(f["name"]))
    assert (version, flags, n) == (1, 3, f["n"])
    assert lock == f["ref_read"]["lock"] and total == len(pl) == f["ref_read"]["states"]


def test_oracle_mixed_rows_and_shuffles(nqsf):
    for f in GOLD["files"]:
        if "mix" in f:
            d1, d2 = f["mix"]
            a, b = nqsf.pool_placements(f["n"], d1), nqsf.pool_placements(f["n"], d2)
            mix = [x for i in range(max(len(a), len(b))) for x in (a[i:i + 1] + b[i:i + 1])]
            assert nqsf.write_bytes(f["n"], d1, mix) == golden_bytes(f["name"])
        elif "-m" in f["args"]:
            n, lock = f["n"], lock_of(f["args"])
            seed = int(f["args"][f["args"].index("-r") + 1]) if "-r" in f["args"] else None
            pool = nqsf.pool_placements(n, lock)
            perm = nqsf.shuffle_perm(len(pool), seed)
            assert nqsf.write_bytes(n, lock, [pool[i] for i in perm]) == golden_bytes(f["name"])


@pytest.mark.parametrize("d", GOLD["dirs"], ids=lambda d: d["name"])
def test_oracle_chunked_files(nqsf, d):
    n, args = d["n"], d["args"]
    lock, chunks = lock_of(args), int(args[args.index("-s") + 1])
    pool = nqsf.pool_placements(n, lock)
    if "-m" in args:
        perm = nqsf.shuffle_perm(len(pool), int(args[args.index("-r") + 1]))
        pool = [pool[i] for i in perm]
    plan = nqsf.chunk_plan(len(pool), chunks, n, "D")
    assert [os.path.basename(p) for p, _, _ in plan] == [c["name"] for c in d["chunks"]]
    for (path, first, size), c in zip(plan, d["chunks"]):
        assert nqsf.write_bytes(n, lock, pool[first:first + size]) == golden_bytes(d["name"], c["name"])


@pytest.mark.parametrize("n", sorted(GOLD["targets"], key=int))
def test_oracle_count_target_sizing(nqsf, n):
    n = int(n)
    for row in GOLD["targets"][str(n)]:
        h = row["h"]
        if "fail_line" in row:
            with pytest.raises(ValueError, match=row["fail_line"]):
                nqsf.target_lock(n, h)
            continue
        lock, count, tried, hit = nqsf.target_lock(n, h)
        if "crash" in row:  # the reference died copying a NULL pool handle
            assert hit and tried[:len(row["tried"])] == row["tried"]
        else:
            assert (lock, count, tried, hit) == (row["lock"], row["count"], row["tried"], False), h


# ---- the library against the oracle and the reference's files ----------------------


@pytest.mark.parametrize("f", R_FILES, ids=lambda f: f["name"])
def test_write_matches_reference_bytes(nqb, f, tmp_path):
    n, lock = f["n"], lock_of(f["args"])
    pl = nqb.generate_pool_placements(n, 2 if lock == 1 else lock)  # lock row 1 holds 2-row states
    out = tmp_path / "w.nqsf"
    nqb.write_state_file(str(out), pl, n, lock)
    assert out.read_bytes() == golden_bytes(f["name"])


@pytest.mark.parametrize("f", GOLD["files"], ids=lambda f: f["name"])
def test_read_reference_files(nqb, nqsf, f):
    info, pl = nqb.read_state_file(os.path.join(NQSF_DIR, f["name"]), expect_n=f["n"])
    _, _, n, lock, total, want = nqsf.read_bytes(golden_bytes(f["name"]))
    assert info == {"version": 1, "flags": 3, "n": n, "locked_row": lock, "count": total}
    assert np.array_equal(pl, placements_array(nqb, n, want))


@pytest.mark.parametrize("f", R_FILES, ids=lambda f: f["name"])
def test_read_states_equal_pool(nqb, f):
    n, lock = f["n"], lock_of(f["args"])
    _, pl = nqb.read_state_file(os.path.join(NQSF_DIR, f["name"]))
    st = nqb.states_from_placements(pl)
    assert st.tobytes() == nqb.generate_pool(n, 2 if lock == 1 else lock).tobytes()


def test_placements_rebuild_pool(nqb):
    for n, d in [(4, 1), (4, 3), (8, 1), (9, 4), (13, 6), (16, 5), (21, 3)]:
        pl = nqb.generate_pool_placements(n, d)
        assert len(pl) == nqb.pool_size(n, d)
        assert nqb.states_from_placements(pl).tobytes() == nqb.generate_pool(n, d).tobytes()
        assert np.all(pl["row"] == d) and np.all(pl["col"][:, d:] == 0xFF)
        w = nqb.states_from_placements(pl, mirror_weight=False)
        assert np.all(w["weight"] == 1)


def test_round_trip_large_pool_and_mixed_rows(nqb, tmp_path):
    pl = nqb.generate_pool_placements(16, 6)
    out = str(tmp_path / "big.nqsf")
    nqb.write_state_file(out, pl, 16, 6)
    assert os.path.getsize(out) == 12 + 10 + 9 + 6 * len(pl)
    info, back = nqb.read_state_file(out, expect_n=16)
    assert info["count"] == len(pl) and np.array_equal(back, pl)
    # mixed rows come back grouped by row, rows ascending, input order kept inside a row
    mix = np.concatenate([nqb.generate_pool_placements(10, 5)[:50], nqb.generate_pool_placements(10, 2)])
    rng = np.random.default_rng(5)
    mix = mix[rng.permutation(len(mix))]
    nqb.write_state_file(out, mix, 10, 2)
    _, back = nqb.read_state_file(out)
    want = np.concatenate([mix[mix["row"] == 2], mix[mix["row"] == 5]])
    assert np.array_equal(back, want)
    # no header
    nqb.write_state_file(out, mix, 10, 2, header=False)
    info, back2 = nqb.read_state_file(out, header=False)
    assert info["version"] == 0 and np.array_equal(back2, want)


@pytest.mark.parametrize("n", sorted(GOLD["targets"], key=int))
def test_count_target_sizing_matches_reference(nqb, n):
    n = int(n)
    for row in GOLD["targets"][str(n)]:
        h = row["h"]
        if "fail_line" in row:
            with pytest.raises(nqb.NQBError) as e:
                nqb.pool_for_target(n, h)
            assert e.value.status == (nqb.E_INVALID if row["fail_line"] == "139" else nqb.E_RANGE)
            continue
        t = nqb.pool_for_target(n, h)
        if "crash" in row:
            assert t["limit_hit"] == 1 and t["tried_count"][:len(row["tried"])] == row["tried"]
            continue
        assert (t["lock_row"], t["count"], t["tried_count"], t["limit_hit"]) == (row["lock"], row["count"],
                                                                                  row["tried"], 0), h
        assert t["pool_depth"] == max(t["lock_row"], 2) and t["hard_limit"] == int(h * 1.2)
        assert nqb.pool_size(n, t["pool_depth"]) == t["count"]


def test_count_target_large_boards(nqb, nqsf):
    """Beyond the fixtures: the library's sizing against the oracle's restatement, and the
    default CLI target (80M states) at N=17 and N=21."""
    for n, h in [(15, 10 ** 5), (16, 3 * 10 ** 5), (16, 12345)]:
        t = nqb.pool_for_target(n, h)
        lock, count, tried, hit = nqsf.target_lock(n, h)
        assert (t["lock_row"], t["count"], t["tried_count"], bool(t["limit_hit"])) == (lock, count, tried, hit)
    t = nqb.pool_for_target(17, 80_000_000)
    assert t["lock_row"] >= 6 and t["count"] <= t["hard_limit"]
    t = nqb.pool_for_target(21, 80_000_000)
    assert (t["lock_row"], t["count"]) == (7, 39430182)


def test_state_file_errors(nqb, tmp_path):
    good = golden_bytes("R_n8_l3.nqsf")
    p = tmp_path / "e.nqsf"

    def status_of(data, **kw):
        p.write_bytes(data)
        with pytest.raises(nqb.NQBError) as e:
            nqb.read_state_file(str(p), **kw)
        return e.value.status

    assert status_of(good[:-1]) == nqb.E_FORMAT                       # truncated states
    assert status_of(good[:30]) == nqb.E_FORMAT                       # truncated segment header
    assert status_of(good[:5]) == nqb.E_FORMAT                        # truncated file header
    assert status_of(b"\x02" + good[1:]) == nqb.E_FORMAT              # version 2 (reader: -3)
    assert status_of(good[:4] + b"\x02" + good[5:]) == nqb.E_FORMAT   # other flags (reader: -4)
    assert status_of(good, expect_n=9) == nqb.E_INVALID               # board size (reader asserts)
    bad_col = bytearray(good); bad_col[-1] = 8
    assert status_of(bytes(bad_col)) == nqb.E_FORMAT                  # column >= n
    bad_row = bytearray(good); bad_row[22] = 8
    assert status_of(bytes(bad_row)) == nqb.E_FORMAT                  # segment row >= n
    more = bytearray(good); more[14] = 71
    assert status_of(bytes(more)) == nqb.E_FORMAT                     # total above the segments
    less = bytearray(good); less[14] = 69
    assert status_of(bytes(less)) == nqb.E_FORMAT                     # segment above the total
    assert status_of(good + b"\x03") == nqb.E_FORMAT                  # trailing partial segment
    with pytest.raises(nqb.NQBError) as e:
        nqb.read_state_file(str(tmp_path / "missing.nqsf"))
    assert e.value.status == nqb.E_IO
    pl = nqb.generate_pool_placements(8, 3)
    for bad in [lambda: nqb.write_state_file(str(p), pl[:0], 8, 3),   # empty: the reference refuses
                lambda: nqb.write_state_file(str(p), pl, 9, 3),        # board size differs
                lambda: nqb.states_from_placements(np.zeros(1, nqb.PLACEMENT_DTYPE))]:
        with pytest.raises(nqb.NQBError) as e:
            bad()
        assert e.value.status == nqb.E_INVALID
    with pytest.raises(nqb.NQBError) as e:
        nqb.write_state_file(str(tmp_path / "no" / "dir.nqsf"), pl, 8, 3)
    assert e.value.status == nqb.E_IO
    for h in [0, 3, 7]:
        with pytest.raises(nqb.NQBError) as e:
            nqb.pool_for_target(8, h)
        assert e.value.status == nqb.E_INVALID


def test_row_zero_states_round_trip(nqb, nqsf, tmp_path):
    """Empty boards (row 0) take no column bytes in a file; they still count toward the
    total, in a segment of their own, and read back as boards with no queen."""
    pl = np.zeros(3, dtype=nqb.PLACEMENT_DTYPE)
    pl["n"], pl["row"], pl["col"] = 9, 0, 0xFF
    mix = np.concatenate([pl, nqb.generate_pool_placements(9, 2)[:4]])
    out = str(tmp_path / "r0.nqsf")
    nqb.write_state_file(out, mix, 9, 0)
    data = open(out, "rb").read()
    assert data == nqsf.write_bytes(9, 0, [(0, [])] * 3 + [(2, list(c[:2])) for c in mix[3:]["col"]])
    info, back = nqb.read_state_file(out)
    assert info["count"] == 7 and np.array_equal(back, mix)
    st = nqb.states_from_placements(back[:3])
    assert np.all(st["cols"] == 0) and np.all(st["weight"] == 1) and np.all(st["row"] == 0)


def test_row_zero_segment_counts_are_bounded(nqb, tmp_path):
    """A row-0 segment carries no column bytes, so the file size cannot bound its count: a
    count whose placement array would not fit (or whose byte size wraps) is a format error,
    not an allocation; a large but plausible count reads back as empty boards."""
    import struct
    good = golden_bytes("R_n8_l3.nqsf")
    p = tmp_path / "z.nqsf"

    def file_with(total, cnt):
        return good[:12] + bytes([8, 0]) + struct.pack("<Q", total) + bytes([0]) + struct.pack("<Q", cnt)

    for cnt in (2 ** 59 + 1, 2 ** 63, 2 ** 32 + 1):
        p.write_bytes(file_with(cnt, cnt))
        with pytest.raises(nqb.NQBError) as e:
            nqb.read_state_file(str(p))
        assert e.value.status == nqb.E_FORMAT, cnt
    p.write_bytes(file_with(1 << 16, 1 << 16))
    info, back = nqb.read_state_file(str(p))
    assert info["count"] == 1 << 16 and len(back) == 1 << 16
    assert np.all(back["row"] == 0) and np.all(back["n"] == 8)
