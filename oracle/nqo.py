"""ctypes binding of the CPU oracle (oracle/nqo.c).  TEST INFRASTRUCTURE ONLY.

Used by tests/, the smoke check and the bench's CPU-baseline leg as the checker; the
product (libnqb.so) never imports it.  The C source cites the reference lines each
function restates (n_queens.cu, GPU_NQueens.cu, diagonals.cuh).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnqo.so")
REF_DIR = os.path.join(HERE, "_ref")

STATE_DTYPE = np.dtype([("cols", "<u4"), ("ldiag", "<u4"), ("rdiag", "<u4"),
                        ("row", "u1"), ("n", "u1"), ("weight", "u1"), ("flags", "u1")])
assert STATE_DTYPE.itemsize == 16

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        L.nqo_pool_size.argtypes = [ctypes.c_uint, ctypes.c_uint, u64p, u64p]
        L.nqo_pool_fill.argtypes = [ctypes.c_uint, ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_uint64, u64p]
        L.nqo_replay_pool.argtypes = [ctypes.c_uint, ctypes.c_uint, ctypes.c_uint64, ctypes.c_uint64,
                                      u64p, u64p, u64p, u64p]
        L.nqo_solve_state.argtypes = [ctypes.c_void_p, u64p, u64p]
        L.nqo_solve_states.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, u64p]
        L.nqo_backtrack_count.argtypes = [ctypes.c_uint, u64p, u64p]
        L.nqo_ref_state_size.argtypes = [ctypes.c_uint]
        L.nqo_ref_state_size.restype = ctypes.c_uint64
        L.nqo_pool_fill_ref.argtypes = [ctypes.c_uint, ctypes.c_uint, ctypes.c_void_p, ctypes.c_uint64, u64p]
        _lib = L
    return _lib


def _u64():
    return ctypes.c_uint64(0)


def pool_size(n, d):
    c, w = _u64(), _u64()
    if lib().nqo_pool_size(n, d, ctypes.byref(c), ctypes.byref(w)):
        raise ValueError(f"bad n/d {n}/{d}")
    return c.value, w.value


def pool(n, d, with_queens=False):
    cnt, _ = pool_size(n, d)
    st = np.zeros(max(cnt, 1), dtype=STATE_DTYPE)
    qs = np.zeros((max(cnt, 1), 32), dtype=np.uint8) if with_queens else None
    got = _u64()
    lib().nqo_pool_fill(n, d, st.ctypes.data, qs.ctypes.data if qs is not None else None, cnt,
                        ctypes.byref(got))
    st = st[:cnt]
    return (st, qs[:cnt]) if with_queens else st


def pool_ref_records(n, d):
    """The pool as reference nq_state_t records (bytes, stride ref_state_size(n))."""
    cnt, _ = pool_size(n, d)
    sz = int(lib().nqo_ref_state_size(n))
    buf = np.zeros(max(cnt, 1) * sz, dtype=np.uint8)
    got = _u64()
    lib().nqo_pool_fill_ref(n, d, buf.ctypes.data, cnt, ctypes.byref(got))
    return buf[:cnt * sz], sz


def pool_hash(n, d):
    """FNV-1a over (curr_row, queen columns) of every state in order, as ref_harness prints."""
    st, qs = pool(n, d, with_queens=True)
    h = 1469598103934665603
    M = (1 << 64) - 1
    for i in range(len(st)):
        r = int(st[i]["row"])
        h = ((h ^ r) * 1099511628211) & M
        for k in range(r):
            h = ((h ^ int(qs[i, k])) * 1099511628211) & M
    return f"{h:016x}"


def replay_pool(n, d, stride=1, offset=0):
    """Kernel-loop replay of the reference over the pool: weighted count, nodes, unit nodes."""
    wc, nd, un, sm = _u64(), _u64(), _u64(), _u64()
    lib().nqo_replay_pool(n, d, stride, offset, ctypes.byref(wc), ctypes.byref(nd), ctypes.byref(un),
                          ctypes.byref(sm))
    return {"count": wc.value, "nodes": nd.value, "unit": un.value, "sampled": sm.value}


def solve_states(states):
    """Independent backtracker over library states: per-state weighted counts, total nodes."""
    states = np.ascontiguousarray(states, dtype=STATE_DTYPE)
    out = np.zeros(max(len(states), 1), dtype=np.uint64)
    tn = _u64()
    lib().nqo_solve_states(states.ctypes.data, len(states), out.ctypes.data, ctypes.byref(tn))
    return out[:len(states)], tn.value


def backtrack_count(n):
    c, nd = _u64(), _u64()
    lib().nqo_backtrack_count(n, ctypes.byref(c), ctypes.byref(nd))
    return c.value, nd.value


def ref_harness_path(n):
    return os.path.join(REF_DIR, f"N{n}", "ref_harness")


def ref_available(n):
    return os.access(ref_harness_path(n), os.X_OK)


def run_ref(n, *args, timeout=None):
    """Runs the reference harness for board n; returns the parsed NQO_JSON lines."""
    import json
    out = subprocess.run([ref_harness_path(n)] + [str(a) for a in args], capture_output=True, text=True,
                         timeout=timeout, check=True).stdout
    return [json.loads(l[len("NQO_JSON "):]) for l in out.splitlines() if l.startswith("NQO_JSON ")]
