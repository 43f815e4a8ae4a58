"""CPU restatement of the reference's state-file format, CLI pool chunking and shuffling,
and count-target pool sizing.  TEST INFRASTRUCTURE ONLY: used by tests/ as the checker;
the product (libnqb.so, the nqb_solver CLI) never imports it.

Placements are (row, columns) pairs: the queens of rows [0, row), as the reference's
nq_state_t holds them in queen_at_index (n_queens.cuh:100-113).
"""
import ctypes
import functools
import math
import struct

import numpy as np

import nqo

FILE_VERSION = 1  # NQ_STATE_FILE_VERSION, nq_utils.cu:13
# util_state_gen_breaking_compilation_flags (nq_utils.cu:65-74) under the reference's default
# build: NQ_ENABLE_EXPERIMENTAL_OPTIMISATIONS (bit 0) and mirror elimination (bit 1) are on.
FILE_FLAGS = 3
PLAY_FACTOR = 0.2  # STATE_GENERATION_LIMIT_PLAY_FACTOR, deffinitions.cuh:61


def write_bytes(n, locked_row, placements, header=True):
    """util_write_nq_states_to_stream (nq_utils.cu:143-194): header, then one segment per
    row present, rows ascending, each with its states in input order."""
    if not placements:
        raise ValueError("the reference writer refuses an empty buffer (nq_utils.cu:193)")
    out = bytearray()
    if header:
        out += struct.pack("<IQ", FILE_VERSION, FILE_FLAGS)
    out += struct.pack("<BBQ", n, locked_row, len(placements))
    rows = {r for r, _ in placements}
    for h in range(n):
        if h in rows:
            seg = [bytes(c[:h]) for r, c in placements if r == h]
            out += struct.pack("<BQ", h, len(seg))
            out += b"".join(seg)
    return bytes(out)


def read_bytes(data, header=True):
    """util_read_nq_states_from_stream (nq_utils.cu:196-252): (version, flags, n, locked_row,
    total, placements).  Raises ValueError where the reference returns -3/-4 or asserts."""
    pos = 0
    version = flags = None
    if header:
        version, flags = struct.unpack_from("<IQ", data, 0)
        pos = 12
        if version != FILE_VERSION or flags != FILE_FLAGS:
            raise ValueError("version or generation flags differ (reader returns -3 / -4)")
    n, lock, total = struct.unpack_from("<BBQ", data, pos)
    pos += 10
    placements = []
    while pos < len(data):
        r = data[pos]
        (cnt,) = struct.unpack_from("<Q", data, pos + 1)
        pos += 9
        if len(placements) + cnt > total or pos + cnt * r > len(data) or r >= n:
            raise ValueError("segment out of bounds (the reference asserts, nq_utils.cu:228-232)")
        for _ in range(cnt):
            cols = list(data[pos:pos + r])
            if any(c >= n for c in cols):
                raise ValueError("column out of range")
            placements.append((r, cols))
            pos += r
    if len(placements) != total:
        raise ValueError("segment counts do not add up to the total")
    return version, flags, n, lock, total, placements


def pool_placements(n, d):
    """The reference's rowlock pool (oracle nqo.pool) as placements; d == 1 gives its
    2-row states, as the reference's generator does."""
    st, qs = nqo.pool(n, d, with_queens=True)
    return [(int(st[i]["row"]), [int(x) for x in qs[i, :st[i]["row"]]]) for i in range(len(st))]


@functools.lru_cache(maxsize=None)
def _sizes(n, lock):
    """Pool size of each row-0 column at lock row `lock` (one generator thread each,
    n_queens.cu:111-124, 157-167); rows >= n hold nothing."""
    half = (n + 1) // 2
    if lock >= n:
        return (0,) * half
    st, qs = nqo.pool(n, lock, with_queens=True)
    return tuple(int(x) for x in np.bincount(qs[:len(st), 0], minlength=half)[:half])


def target_lock(n, how_many):
    """gen_states_threaded (n_queens.cu:128-219): (lock_row, count, tried_counts, limit_hit).
    Raises ValueError where the reference fails (lock row 0, n_queens.cu:139; no row within
    the limit, :196).  When one column's pool reaches the hard limit the reference's thread
    returns NULL and the process crashes copying it (:118-119); the restatement follows the
    error path the code means (:176-180): stop with the previous row, limit_hit = True."""
    hard = int(how_many * (1 + PLAY_FACTOR))
    lock = int(math.log(how_many) / math.log(n))
    lock = n - 1 if lock >= n else lock
    if lock == 0:
        raise ValueError("lock row 0 (n_queens.cu:139)")
    actual = None
    tmp = None
    tried = []
    limit_hit = False
    while True:
        actual = tmp
        per = _sizes(n, lock)
        tried.append(sum(per))
        if any(p >= hard for p in per):
            limit_hit = True
            break
        tmp = (lock, sum(per))
        lock += 1
        if not (tmp[1] >= (actual[1] if actual else 0) and lock <= n and tmp[1] <= hard):
            break
    if actual is None:
        raise ValueError("no lock row within the hard limit (n_queens.cu:196)")
    return actual[0], actual[1], tried, limit_hit


def _libc():
    return ctypes.CDLL(None)


def shuffle_perm(length, seed=None):
    """shuffle_states (NQ_solver.cu:40-55) as a permutation: result[i] = the input index of
    the state that ends at position i.  Uses the C library's rand(), seeded by srand(seed)
    as `-r` does (NQ_solver.cu:268-273); without `-r`, rand() starts as after srand(1)
    (the C standard's initial state)."""
    libc = _libc()
    libc.srand(ctypes.c_uint(1 if seed is None else seed))
    perm = list(range(length))
    if length < 3:
        return perm
    for i in range(length - 2):
        words = [libc.rand() & 0xFFFF for _ in range(4)]  # int16_t lanes of a uint64 union
        rval = words[0] | words[1] << 16 | words[2] << 32 | words[3] << 48
        rval = ((rval % length) + i) % length
        if rval == i:
            continue
        perm[i], perm[rval] = perm[rval], perm[i]
    return perm


def chunk_plan(count, chunks, n, out_dir):
    """write_gen_states_to_file (NQ_solver.cu:57-108): [(path, first, size)] per chunk file."""
    per = math.ceil(count / chunks)
    if not per:
        raise ValueError("more chunks than states")
    left = count % chunks
    plan, written = [], 0
    for i in range(chunks):
        plan.append((f"{out_dir}/chunk_{i}_for_n{n}_cnt_{per}.nqsf", written, per))
        written += per
        if i == left - 1:
            per -= 1
    return plan
