"""Python binding of libnqb.so, the B200 N-Queens counter (C ABI in include/nqb.h).

Mirrors the reference's host calls (fillpant/GPU-N-Queens):
  count(n, depth)            nq_generate_states_rowlock + solve()/gpu_solver_driver
                             (n_queens.cuh:119, NQ_solver.cu:192-209, GPU_NQueens.cuh:13)
  generate_pool(n, depth)    nq_generate_states_rowlock (n_queens.cuh:119)
  solve_ref_states(...)      gpu_solver_driver on reference nq_state_t records
The reference aborts on errors (FAIL_IF / CHECK_CUDA_ERROR, deffinitions.cuh:148-156);
here every failure raises NQBError carrying the library's status code.  There is no
CPU fallback: if libnqb.so is missing, loading raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# NQB_LIBRARY selects another build of the same C ABI, e.g. the bounds-checked
# libnqb_checked.so (`make -C gpu-n-queens_b200 checked`)
LIB_PATH = os.environ.get("NQB_LIBRARY") or os.path.join(HERE, "libnqb.so")
INCLUDE_DIR = os.path.join(os.path.dirname(HERE), "include")

STATE_DTYPE = np.dtype([("cols", "<u4"), ("ldiag", "<u4"), ("rdiag", "<u4"),
                        ("row", "u1"), ("n", "u1"), ("weight", "u1"), ("flags", "u1")])
assert STATE_DTYPE.itemsize == 16

OK, E_INVALID, E_NOMEM, E_CUDA, E_NODEVICE, E_RANGE, E_STALL, E_DEVICE, E_MODEL, E_IO, E_FORMAT = range(11)
PLACEMENT_DTYPE = np.dtype([("n", "u1"), ("row", "u1"), ("col", "u1", (30,))])
assert PLACEMENT_DTYPE.itemsize == 32
STATE_FILE_VERSION, STATE_FILE_FLAGS = 1, 3
FORM_PLAIN, FORM_BATCHED = 0, 1
MIN_N, MAX_N = 4, 31


class NQBError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        super().__init__(f"{what}: {strerror(status)} (status {status})" if what else strerror(status))


class Opts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("form", ctypes.c_int), ("block_size", ctypes.c_int),
                ("count_unit_nodes", ctypes.c_int), ("max_split_rounds", ctypes.c_int),
                ("split_factor", ctypes.c_int), ("model", ctypes.c_void_p), ("host_pool", ctypes.c_int),
                ("autotune", ctypes.c_int), ("count_lane_steps", ctypes.c_int), ("sched_cost", ctypes.c_int),
                ("reserved", ctypes.c_int * 4)]


class Stats(ctypes.Structure):
    _fields_ = [("states", ctypes.c_uint64), ("nodes", ctypes.c_uint64), ("unit_nodes", ctypes.c_uint64),
                ("gen_ms", ctypes.c_double), ("h2d_ms", ctypes.c_double), ("kernel_ms", ctypes.c_double),
                ("wall_ms", ctypes.c_double), ("pregen_depth", ctypes.c_uint32),
                ("kernel_launches", ctypes.c_uint32), ("items", ctypes.c_uint64), ("sched_ms", ctypes.c_double),
                ("block_size", ctypes.c_uint32), ("form", ctypes.c_int32), ("placed_lane_steps", ctypes.c_uint64),
                ("lane_step_slots", ctypes.c_uint64)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}
        if d["unit_nodes"] == 2 ** 64 - 1:
            d["unit_nodes"] = None
        d["lane_efficiency"] = (self.placed_lane_steps / self.lane_step_slots) if self.lane_step_slots else None
        return d


_lib = None


def build():
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    """Loads libnqb.so (raises OSError when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: run `make -C {HERE}` (there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        vp = ctypes.c_void_p
        sig = {
            "nqb_default_opts": (None, [ctypes.POINTER(Opts)]),
            "nqb_strerror": (ctypes.c_char_p, [ctypes.c_int]),
            "nqb_version": (ctypes.c_int, []),
            "nqb_device_check": (ctypes.c_int, [ctypes.c_int]),
            "nqb_count": (ctypes.c_int, [ctypes.c_uint, ctypes.c_uint, u64p]),
            "nqb_count_ex": (ctypes.c_int, [ctypes.c_uint, ctypes.c_uint, ctypes.POINTER(Opts), u64p,
                                            ctypes.POINTER(Stats)]),
            "nqb_generate_pool": (ctypes.c_int, [ctypes.c_uint, ctypes.c_uint, ctypes.POINTER(vp), u64p]),
            "nqb_generate_pool_into": (ctypes.c_int, [ctypes.c_uint, ctypes.c_uint, vp, ctypes.c_uint64, u64p]),
            "nqb_pool_weighted_size": (ctypes.c_int, [ctypes.c_uint, ctypes.c_uint, u64p]),
            "nqb_free": (None, [vp]),
            "nqb_solve_states": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.POINTER(Opts), u64p,
                                                ctypes.POINTER(Stats)]),
            "nqb_solve_batch": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.POINTER(Opts), vp,
                                               ctypes.POINTER(Stats)]),
            "nqb_ref_state_size": (ctypes.c_size_t, [ctypes.c_uint]),
            "nqb_states_from_ref": (ctypes.c_int, [ctypes.c_uint, vp, ctypes.c_uint64, ctypes.c_int, vp]),
            "nqb_solve_ref_states": (ctypes.c_int, [ctypes.c_uint, vp, ctypes.c_uint64, ctypes.c_uint,
                                                    ctypes.POINTER(Opts), u64p]),
            "nqb_sample_boards": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint, ctypes.c_uint,
                                                 ctypes.c_uint, ctypes.c_uint, vp]),
            "nqb_plain_launch": (ctypes.c_int, [vp, ctypes.c_uint64, vp, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_uint, vp]),
            "nqb_batched_launch": (ctypes.c_int, [vp, ctypes.c_uint64, vp, vp, vp, ctypes.c_int, ctypes.c_uint,
                                                  vp]),
            "nqb_batched_launch_ex": (ctypes.c_int, [vp, ctypes.c_uint64, vp, vp, ctypes.c_uint64, vp, vp,
                                                     ctypes.c_int, ctypes.c_uint, ctypes.c_uint, vp]),
            "nqb_generate_pool_placements": (ctypes.c_int, [ctypes.c_uint, ctypes.c_uint, ctypes.POINTER(vp), u64p]),
            "nqb_states_from_placements": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.c_int, vp]),
            "nqb_write_state_file": (ctypes.c_int, [ctypes.c_char_p, vp, ctypes.c_uint64, ctypes.c_uint,
                                                    ctypes.c_uint, ctypes.c_int]),
            "nqb_read_state_file": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_uint,
                                                   ctypes.POINTER(StateFileInfo), ctypes.POINTER(vp)]),
            "nqb_pool_for_target": (ctypes.c_int, [ctypes.c_uint, ctypes.c_uint64, ctypes.POINTER(Target)]),
            "nqb_tune_count": (ctypes.c_int, [ctypes.c_uint, vp, ctypes.c_uint, ctypes.POINTER(Opts), ctypes.c_uint,
                                              ctypes.POINTER(TuneResult)]),
            "nqb_solve_states_multi": (ctypes.c_int, [vp, ctypes.c_uint64, vp, ctypes.c_uint, ctypes.POINTER(Opts),
                                                      u64p, ctypes.POINTER(Stats)]),
            "nqb_device_count": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int)]),
            "nqb_trim_device_memory": (ctypes.c_int, [ctypes.c_int]),
            "nqb_debug_fail_allocation": (ctypes.c_longlong, [ctypes.c_longlong]),
            "nqb_measure_int32_peak": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                                      ctypes.POINTER(ctypes.c_double)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def strerror(status):
    try:
        return lib().nqb_strerror(status).decode()
    except OSError:
        return f"status {status}"


def _check(status, what):
    if status != OK:
        raise NQBError(status, what)


def make_opts(device=0, form=FORM_PLAIN, block_size=0, count_unit_nodes=False, model=None, max_split_rounds=-1,
              split_factor=0, host_pool=False, autotune=False, count_lane_steps=False, sched_cost=0):
    o = Opts()
    lib().nqb_default_opts(ctypes.byref(o))
    o.device, o.form, o.block_size = device, form, block_size
    o.count_unit_nodes, o.max_split_rounds, o.split_factor = int(count_unit_nodes), max_split_rounds, split_factor
    o.model = model.handle if model is not None else None
    o.host_pool = int(host_pool)
    o.autotune = int(autotune)
    o.count_lane_steps = int(count_lane_steps)
    o.sched_cost = int(sched_cost)
    return o


def device_check(device=0):
    return lib().nqb_device_check(device)


def count(n, depth, **opts):
    """Mirror-weighted number of n-queens solutions via a depth-row pool (the drop-in)."""
    c = ctypes.c_uint64(0)
    _check(lib().nqb_count_ex(n, depth, ctypes.byref(make_opts(**opts)), ctypes.byref(c), None),
           f"nqb_count({n}, {depth})")
    return c.value


def count_ex(n, depth, **opts):
    """(count, stats dict) for the (n, depth) pool."""
    c = ctypes.c_uint64(0)
    st = Stats()
    _check(lib().nqb_count_ex(n, depth, ctypes.byref(make_opts(**opts)), ctypes.byref(c), ctypes.byref(st)),
           f"nqb_count_ex({n}, {depth})")
    return c.value, st.as_dict()


def pool_size(n, depth):
    c = ctypes.c_uint64(0)
    _check(lib().nqb_generate_pool_into(n, depth, None, 0, ctypes.byref(c)), "nqb_generate_pool_into")
    return c.value


def pool_weighted_size(n, depth):
    w = ctypes.c_uint64(0)
    _check(lib().nqb_pool_weighted_size(n, depth, ctypes.byref(w)), "nqb_pool_weighted_size")
    return w.value


def generate_pool(n, depth):
    """The (n, depth) pool as a numpy array of STATE_DTYPE, in the reference's order."""
    cnt = pool_size(n, depth)
    out = np.zeros(max(cnt, 1), dtype=STATE_DTYPE)
    got = ctypes.c_uint64(0)
    _check(lib().nqb_generate_pool_into(n, depth, out.ctypes.data, cnt, ctypes.byref(got)), "nqb_generate_pool_into")
    return out[:got.value]


def generate_pool_device(n, depth):
    """The pool built on the GPU (nqb_generate_pool_device_into), returned as a numpy array."""
    import torch
    L = lib()
    vp = ctypes.c_void_p
    f = L.nqb_generate_pool_device_into
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_uint, ctypes.c_uint, vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64), vp]
    cap = pool_size(n, depth)
    buf = torch.empty(max(cap, 1) * 16, dtype=torch.uint8, device="cuda")
    c = ctypes.c_uint64(0)
    _check(f(n, depth, buf.data_ptr(), cap, ctypes.byref(c), torch.cuda.current_stream().cuda_stream),
           "nqb_generate_pool_device_into")
    torch.cuda.synchronize()
    return buf[:16 * c.value].cpu().numpy().view(STATE_DTYPE)


def _take(ptr, nbytes):
    """Copies a library allocation into Python bytes and releases it with nqb_free."""
    try:
        return bytes((ctypes.c_uint8 * nbytes).from_address(ptr.value)) if nbytes else b""
    finally:
        lib().nqb_free(ptr)


def generate_pool_placements(n, depth):
    """The (n, depth) pool as placements (PLACEMENT_DTYPE), same states and order as generate_pool."""
    p = ctypes.c_void_p()
    c = ctypes.c_uint64(0)
    _check(lib().nqb_generate_pool_placements(n, depth, ctypes.byref(p), ctypes.byref(c)),
           "nqb_generate_pool_placements")
    return np.frombuffer(_take(p, 32 * c.value), dtype=PLACEMENT_DTYPE).copy()


def states_from_placements(placements, mirror_weight=True):
    pl = np.ascontiguousarray(placements, dtype=PLACEMENT_DTYPE)
    out = np.zeros(max(len(pl), 1), dtype=STATE_DTYPE)
    _check(lib().nqb_states_from_placements(pl.ctypes.data, len(pl), int(mirror_weight), out.ctypes.data),
           "nqb_states_from_placements")
    return out[:len(pl)]


class StateFileInfo(ctypes.Structure):
    _fields_ = [("version", ctypes.c_uint32), ("flags", ctypes.c_uint64), ("n", ctypes.c_uint),
                ("locked_row", ctypes.c_uint), ("count", ctypes.c_uint64)]


def write_state_file(path, placements, n, locked_row, header=True):
    pl = np.ascontiguousarray(placements, dtype=PLACEMENT_DTYPE)
    _check(lib().nqb_write_state_file(os.fsencode(path), pl.ctypes.data, len(pl), n, locked_row, int(header)),
           f"nqb_write_state_file({path})")


def read_state_file(path, header=True, expect_n=0):
    """(info dict, placements) of a .nqsf state file."""
    info = StateFileInfo()
    p = ctypes.c_void_p()
    _check(lib().nqb_read_state_file(os.fsencode(path), int(header), expect_n, ctypes.byref(info), ctypes.byref(p)),
           f"nqb_read_state_file({path})")
    pl = np.frombuffer(_take(p, 32 * info.count), dtype=PLACEMENT_DTYPE).copy()
    return {k: getattr(info, k) for k, _ in StateFileInfo._fields_}, pl


class TuneEntry(ctypes.Structure):
    _fields_ = [("depth", ctypes.c_uint), ("form", ctypes.c_int), ("block_size", ctypes.c_int),
                ("split_factor", ctypes.c_int), ("ms", ctypes.c_double)]


class TuneResult(ctypes.Structure):
    _fields_ = [("depth", ctypes.c_uint), ("form", ctypes.c_int), ("block_size", ctypes.c_int),
                ("split_factor", ctypes.c_int), ("best_ms", ctypes.c_double), ("sample_states", ctypes.c_uint64),
                ("sample_div", ctypes.c_uint), ("n_tried", ctypes.c_uint), ("tried", TuneEntry * 64)]


def tune_count(n, depths, sample_div=64, **opts):
    """Launch autotuner (nqb_tune_count): the fastest (depth, form, block size, split factor)
    on a 1/sample_div stride sample of each depth's pool, with every candidate's time."""
    if isinstance(depths, int):
        depths = [depths]
    ds = (ctypes.c_uint * len(depths))(*depths)
    r = TuneResult()
    _check(lib().nqb_tune_count(n, ds, len(depths), ctypes.byref(make_opts(**opts)), sample_div, ctypes.byref(r)),
           f"nqb_tune_count({n}, {list(depths)})")
    keys = ("depth", "form", "block_size", "split_factor")
    return {**{k: getattr(r, k) for k in keys}, "best_ms": r.best_ms, "sample_states": r.sample_states,
            "sample_div": r.sample_div,
            "tried": [{**{k: getattr(e, k) for k in keys}, "ms": round(e.ms, 3)} for e in r.tried[:r.n_tried]]}


class Target(ctypes.Structure):
    _fields_ = [("lock_row", ctypes.c_uint), ("pool_depth", ctypes.c_uint), ("count", ctypes.c_uint64),
                ("hard_limit", ctypes.c_uint64), ("first_row", ctypes.c_uint), ("tried", ctypes.c_uint),
                ("limit_hit", ctypes.c_int), ("reserved", ctypes.c_uint), ("tried_count", ctypes.c_uint64 * 32)]


def pool_for_target(n, how_many):
    """Count-target sizing: dict with lock_row, pool_depth, count, hard_limit, first_row, tried rows."""
    t = Target()
    _check(lib().nqb_pool_for_target(n, ctypes.c_uint64(how_many), ctypes.byref(t)),
           f"nqb_pool_for_target({n}, {how_many})")
    d = {k: getattr(t, k) for k, _ in Target._fields_ if k not in ("reserved", "tried_count")}
    d["tried_count"] = list(t.tried_count[:t.tried])
    return d


def solve_states_multi(states, devices, **opts):
    """(total, stats) of host states split in contiguous slices across `devices`."""
    states = np.ascontiguousarray(states, dtype=STATE_DTYPE)
    devs = (ctypes.c_int * len(devices))(*devices)
    t = ctypes.c_uint64(0)
    st = Stats()
    _check(lib().nqb_solve_states_multi(states.ctypes.data, len(states), devs, len(devices),
                                        ctypes.byref(make_opts(**opts)), ctypes.byref(t), ctypes.byref(st)),
           "nqb_solve_states_multi")
    return t.value, st.as_dict()


def measure_int32_peak(device=0):
    """(best, {kind: lane-ops/s}) of the INT32 issue-rate microbenchmark."""
    best = ctypes.c_double(0)
    kinds = (ctypes.c_double * 4)()
    _check(lib().nqb_measure_int32_peak(device, ctypes.byref(best), kinds), "nqb_measure_int32_peak")
    return best.value, dict(zip(("lop3", "add", "imad", "lop3_imad"), list(kinds)))


def trim_device_memory(device=0):
    """Returns the library's cached device memory on `device` to the driver."""
    _check(lib().nqb_trim_device_memory(device), "nqb_trim_device_memory")


def debug_fail_allocation(after):
    """Test hook (nqb_debug_fail_allocation): the library's next `after` allocations succeed and
    the one after them fails as out of memory; a negative value turns the hook off.  Returns the
    countdown it replaces (-1: the hook was off or has fired)."""
    return int(lib().nqb_debug_fail_allocation(after))


def device_count():
    c = ctypes.c_int(0)
    status = lib().nqb_device_count(ctypes.byref(c))
    return c.value if status == OK else 0


def generate_pool_alloc(n, depth):
    """Same pool through nqb_generate_pool (library-allocated, released with nqb_free)."""
    p = ctypes.c_void_p()
    c = ctypes.c_uint64(0)
    _check(lib().nqb_generate_pool(n, depth, ctypes.byref(p), ctypes.byref(c)), "nqb_generate_pool")
    try:
        buf = (ctypes.c_uint8 * (16 * c.value)).from_address(p.value) if c.value else b""
        return np.frombuffer(bytes(buf), dtype=STATE_DTYPE).copy()
    finally:
        lib().nqb_free(p)


def solve_states(states, **opts):
    """(total, stats) for library states in host memory."""
    states = np.ascontiguousarray(states, dtype=STATE_DTYPE)
    t = ctypes.c_uint64(0)
    st = Stats()
    _check(lib().nqb_solve_states(states.ctypes.data if len(states) else None, len(states),
                                  ctypes.byref(make_opts(**opts)), ctypes.byref(t), ctypes.byref(st)),
           "nqb_solve_states")
    return t.value, st.as_dict()


def solve_batch(boards, **opts):
    """(per-board weighted counts as uint64 array, stats)."""
    boards = np.ascontiguousarray(boards, dtype=STATE_DTYPE)
    out = np.zeros(max(len(boards), 1), dtype=np.uint64)
    st = Stats()
    _check(lib().nqb_solve_batch(boards.ctypes.data if len(boards) else None, len(boards),
                                 ctypes.byref(make_opts(**opts)), out.ctypes.data, ctypes.byref(st)),
           "nqb_solve_batch")
    return out[:len(boards)], st.as_dict()


BATCH_SEED = 0x4E51554545534231  # uneven partial boards: 65,536 boards, n 16..20, depth 3..7
MODEL_SEED = 0x4E5131384C524E31  # cost-model training set: n = 18, depth 4..8


def sample_boards(seed, count, n_min, n_max, d_min, d_max):
    """Seeded random valid partial boards (see nqb_sample_boards)."""
    out = np.zeros(max(count, 1), dtype=STATE_DTYPE)
    _check(lib().nqb_sample_boards(seed, count, n_min, n_max, d_min, d_max, out.ctypes.data), "nqb_sample_boards")
    return out[:count]


def ref_state_size(n):
    return int(lib().nqb_ref_state_size(n))


def states_from_ref(n, ref_bytes, mirror_weight=True):
    sz = ref_state_size(n)
    ref_bytes = np.ascontiguousarray(np.frombuffer(ref_bytes, dtype=np.uint8))
    cnt = len(ref_bytes) // sz
    out = np.zeros(max(cnt, 1), dtype=STATE_DTYPE)
    _check(lib().nqb_states_from_ref(n, ref_bytes.ctypes.data, cnt, int(mirror_weight), out.ctypes.data),
           "nqb_states_from_ref")
    return out[:cnt]


def solve_ref_states(n, ref_bytes, locked_row, **opts):
    """gpu_solver_driver replacement on reference nq_state_t records."""
    sz = ref_state_size(n)
    ref_bytes = np.ascontiguousarray(np.frombuffer(ref_bytes, dtype=np.uint8))
    t = ctypes.c_uint64(0)
    _check(lib().nqb_solve_ref_states(n, ref_bytes.ctypes.data, len(ref_bytes) // sz, locked_row,
                                      ctypes.byref(make_opts(**opts)), ctypes.byref(t)), "nqb_solve_ref_states")
    return t.value


def plain_launch(d_states_ptr, count, d_out_ptr, block_size=0, count_unit_nodes=False, stack_depth=0,
                 stream=0):
    """Launches the plain kernel on device pointers (see nqb_plain_launch)."""
    _check(lib().nqb_plain_launch(d_states_ptr, count, d_out_ptr, block_size, int(count_unit_nodes),
                                  stack_depth, stream or None), "nqb_plain_launch")


def batched_launch(d_items_ptr, count, d_head_ptr, d_out_ptr, d_order_ptr=None, block_size=0, stack_depth=0,
                   stream=0):
    """Launches the batched (persistent, work-queue) kernel on device pointers."""
    _check(lib().nqb_batched_launch(d_items_ptr, count, d_order_ptr, d_head_ptr, d_out_ptr, block_size,
                                    stack_depth, stream or None), "nqb_batched_launch")


BATCHED_SCRATCH_BYTES = 64 + 32 * 65536  # NQB_BATCHED_SCRATCH_BYTES


def batched_launch_ex(d_items_ptr, count, d_scratch_ptr, scratch_bytes, d_out_ptr, d_order_ptr=None,
                      d_lane_stats_ptr=None, block_size=0, stack_depth=0, wait_limit=0, stream=0):
    """Launches the batched kernel with work stealing across warps (see nqb_batched_launch_ex);
    the caller reads the launch's error flags from d_out[3]."""
    _check(lib().nqb_batched_launch_ex(d_items_ptr, count, d_order_ptr, d_scratch_ptr, scratch_bytes, d_out_ptr,
                                       d_lane_stats_ptr, block_size, stack_depth, wait_limit, stream or None),
           "nqb_batched_launch_ex")


MODEL_INPUTS, MODEL_PARAMS = 112, 31105


class TrainOpts(ctypes.Structure):
    _fields_ = [("epochs", ctypes.c_int), ("batch", ctypes.c_int), ("lr", ctypes.c_float),
                ("reserved0", ctypes.c_int), ("seed", ctypes.c_uint64), ("reserved", ctypes.c_int * 8)]


def _model_sigs(L):
    vp, fp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)
    sig = {
        "nqb_model_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(vp)]),
        "nqb_model_destroy": (None, [vp]),
        "nqb_model_get_params": (ctypes.c_int, [vp, vp]),
        "nqb_model_set_params": (ctypes.c_int, [vp, vp]),
        "nqb_model_features": (ctypes.c_int, [vp, ctypes.c_uint64, vp]),
        "nqb_model_predict": (ctypes.c_int, [vp, vp, ctypes.c_uint64, vp]),
        "nqb_model_predict_ex": (ctypes.c_int, [vp, vp, ctypes.c_uint64, vp, ctypes.c_uint32]),
        "nqb_model_loss_grad": (ctypes.c_int, [vp, vp, vp, ctypes.c_uint64, fp, vp]),
        "nqb_model_train": (ctypes.c_int, [vp, vp, vp, ctypes.c_uint64, ctypes.POINTER(TrainOpts), vp]),
        "nqb_record_nodes": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.POINTER(Opts), vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype, f.argtypes = res, args


class Model:
    """The learned cost model (nqb_model_*): predicts log2(1 + nodes) below a state."""

    def __init__(self, device=0, seed=1):
        L = lib()
        _model_sigs(L)
        h = ctypes.c_void_p()
        _check(L.nqb_model_create(device, seed, ctypes.byref(h)), "nqb_model_create")
        self.handle, self.device = h.value, device

    def close(self):
        if self.handle:
            lib().nqb_model_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_params(self):
        p = np.zeros(MODEL_PARAMS, dtype=np.float32)
        _check(lib().nqb_model_get_params(self.handle, p.ctypes.data), "nqb_model_get_params")
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == MODEL_PARAMS
        _check(lib().nqb_model_set_params(self.handle, p.ctypes.data), "nqb_model_set_params")

    def predict(self, states, wait_limit=0):
        """Predicted log2(1 + nodes) per state.  wait_limit bounds each tensor-core completion
        wait (0: the library default); a wait that runs out raises NQBError(E_STALL)."""
        states = np.ascontiguousarray(states, dtype=STATE_DTYPE)
        out = np.zeros(max(len(states), 1), dtype=np.float32)
        _check(lib().nqb_model_predict_ex(self.handle, states.ctypes.data, len(states), out.ctypes.data, wait_limit),
               "nqb_model_predict_ex")
        return out[:len(states)]

    def loss_grad(self, states, targets):
        states = np.ascontiguousarray(states, dtype=STATE_DTYPE)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        g = np.zeros(MODEL_PARAMS, dtype=np.float32)
        loss = ctypes.c_float(0)
        _check(lib().nqb_model_loss_grad(self.handle, states.ctypes.data, t.ctypes.data, len(states),
                                         ctypes.byref(loss), g.ctypes.data), "nqb_model_loss_grad")
        return loss.value, g

    def train(self, states, targets, epochs=8, batch=4096, lr=1e-3, seed=1):
        states = np.ascontiguousarray(states, dtype=STATE_DTYPE)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        o = TrainOpts(epochs=epochs, batch=batch, lr=lr, seed=seed)
        losses = np.zeros(epochs, dtype=np.float32)
        _check(lib().nqb_model_train(self.handle, states.ctypes.data, t.ctypes.data, len(states), ctypes.byref(o),
                                     losses.ctypes.data), "nqb_model_train")
        return losses


def model_features(states):
    L = lib()
    _model_sigs(L)
    states = np.ascontiguousarray(states, dtype=STATE_DTYPE)
    out = np.zeros((max(len(states), 1), MODEL_INPUTS), dtype=np.float32)
    _check(L.nqb_model_features(states.ctypes.data, len(states), out.ctypes.data), "nqb_model_features")
    return out[:len(states)]


class BatchPlan:
    """A board set solved repeatedly through one captured CUDA graph (nqb_batch_plan_*)."""

    def __init__(self, boards, device=0, model=None, autotune=True, block_size=0, split_factor=0,
                 max_split_rounds=-1, sched_cost=0):
        L = lib()
        vp = ctypes.c_void_p
        for name, (res, args) in {
            "nqb_batch_plan_create": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.POINTER(Opts), ctypes.c_int,
                                                     ctypes.POINTER(vp)]),
            "nqb_batch_plan_run": (ctypes.c_int, [vp, vp, ctypes.POINTER(Stats)]),
            "nqb_batch_plan_config": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                                     ctypes.POINTER(ctypes.c_uint64)]),
            "nqb_batch_plan_destroy": (None, [vp]),
        }.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        self.handle = None
        self.boards = np.ascontiguousarray(boards, dtype=STATE_DTYPE)
        o = make_opts(device=device, form=FORM_BATCHED, block_size=block_size, model=model,
                      max_split_rounds=max_split_rounds, split_factor=split_factor, sched_cost=sched_cost)
        h = ctypes.c_void_p()
        _check(L.nqb_batch_plan_create(self.boards.ctypes.data, len(self.boards), ctypes.byref(o), int(autotune),
                                       ctypes.byref(h)), "nqb_batch_plan_create")
        self.handle = h.value

    def run(self):
        out = np.zeros(len(self.boards), dtype=np.uint64)
        st = Stats()
        _check(lib().nqb_batch_plan_run(self.handle, out.ctypes.data, ctypes.byref(st)), "nqb_batch_plan_run")
        return out, st.as_dict()

    def config(self):
        b, f, n = ctypes.c_int(), ctypes.c_int(), ctypes.c_uint64()
        _check(lib().nqb_batch_plan_config(self.handle, ctypes.byref(b), ctypes.byref(f), ctypes.byref(n)),
               "nqb_batch_plan_config")
        return {"block_size": b.value, "split_factor": f.value, "items": n.value}

    def close(self):
        if self.handle:
            lib().nqb_batch_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def record_nodes(states, device=0):
    """(nodes, weighted counts) per state, recorded by the batched search kernel."""
    L = lib()
    _model_sigs(L)
    states = np.ascontiguousarray(states, dtype=STATE_DTYPE)
    nodes = np.zeros(max(len(states), 1), dtype=np.uint64)
    counts = np.zeros(max(len(states), 1), dtype=np.uint64)
    _check(L.nqb_record_nodes(states.ctypes.data, len(states), ctypes.byref(make_opts(device=device)),
                              nodes.ctypes.data, counts.ctypes.data), "nqb_record_nodes")
    return nodes[:len(states)], counts[:len(states)]


def header_symbols():
    """Names of the functions include/nqb.h declares."""
    import re
    src = open(os.path.join(INCLUDE_DIR, "nqb.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(nqb_[a-z0-9_]+)\s*\(", src)))
