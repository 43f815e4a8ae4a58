"""The C ABI: libnqb.so loads, exports every function include/nqb.h declares, and rejects bad
arguments with status codes (never exiting).  No GPU needed: no compute call is made."""
import ctypes
import os
import subprocess

import pytest


def test_library_loads_and_exports_header(nqb):
    L = nqb.lib()
    syms = nqb.header_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(L, s), s
    dyn = subprocess.run(["nm", "-D", "--defined-only", nqb.LIB_PATH], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in dyn.splitlines() if " T " in l}
    assert set(syms) <= exported


def test_version_and_strerror(nqb):
    assert nqb.lib().nqb_version() == 10200
    for s in range(9):
        assert nqb.strerror(s) not in ("", "unknown status")
    assert nqb.strerror(99) == "unknown status"


def test_invalid_arguments_return_status(nqb):
    L = nqb.lib()
    c = ctypes.c_uint64(0)
    assert L.nqb_count(3, 1, ctypes.byref(c)) == nqb.E_INVALID
    assert L.nqb_count(32, 4, ctypes.byref(c)) == nqb.E_INVALID
    assert L.nqb_count(12, 0, ctypes.byref(c)) == nqb.E_INVALID
    assert L.nqb_count(12, 12, ctypes.byref(c)) == nqb.E_INVALID
    assert L.nqb_count(12, 4, None) == nqb.E_INVALID
    assert L.nqb_solve_states(None, 5, None, ctypes.byref(c), None) == nqb.E_INVALID
    assert L.nqb_solve_states(None, 0, None, ctypes.byref(c), None) == nqb.OK and c.value == 0
    assert L.nqb_solve_ref_states(12, None, 5, 3, None, ctypes.byref(c)) == nqb.E_INVALID
    assert L.nqb_solve_ref_states(12, None, 0, 0, None, ctypes.byref(c)) == nqb.E_INVALID
    assert L.nqb_plain_launch(None, 10, None, 0, 0, 0, None) == nqb.E_INVALID
    assert L.nqb_plain_launch(None, 0, ctypes.byref(c), 0, 0, 0, None) == nqb.OK


def test_unknown_block_size_rejected(nqb):
    c = ctypes.c_uint64(0)
    assert nqb.lib().nqb_plain_launch(ctypes.c_void_p(16), 1, ctypes.byref(c), 96, 0, 4, None) == nqb.E_INVALID


def test_no_device_reports_nodevice(nqb):
    if nqb.device_check(0) == nqb.OK:
        pytest.skip("a usable GPU is present")
    c = ctypes.c_uint64(0)
    assert nqb.lib().nqb_count(10, 3, ctypes.byref(c)) == nqb.E_NODEVICE


def test_default_opts(nqb):
    o = nqb.make_opts()
    assert (o.device, o.form, o.block_size, o.count_unit_nodes, o.max_split_rounds, o.split_factor) == (0, 0, 0, 0, -1, 0)
    assert not o.model


def test_struct_layouts_match_header(nqb, tmp_path):
    """Every ctypes structure of the binding has the header's size and field offsets (a C
    program compiled against include/nqb.h prints them)."""
    from conftest import ROOT
    structs = {"nqb_opts": nqb.Opts, "nqb_stats": nqb.Stats, "nqb_state_file": nqb.StateFileInfo,
               "nqb_target": nqb.Target, "nqb_tune_entry": nqb.TuneEntry, "nqb_tune_result": nqb.TuneResult}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "nqb.h"', "int main(void) {"]
    for cname, cls in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in cls._fields_:
            lines.append(f'printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines += ['printf("nqb_placement size %zu\\n", sizeof(nqb_placement));',
              'printf("nqb_state size %zu\\n", sizeof(nqb_state));', "return 0; }"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        name, field, val = line.split()
        got[(name, field)] = int(val)
    for cname, cls in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for f in cls._fields_:
            assert got[(cname, f[0])] == getattr(cls, f[0]).offset, (cname, f[0])
    assert got[("nqb_placement", "size")] == nqb.PLACEMENT_DTYPE.itemsize == 32
    assert got[("nqb_state", "size")] == nqb.STATE_DTYPE.itemsize == 16


def test_new_entry_points_reject_bad_arguments_without_a_device(nqb):
    """Argument checks come before any device work, so they answer on a machine without a
    GPU as on a B200."""
    L = nqb.lib()
    u64 = ctypes.c_uint64()
    vp = ctypes.c_void_p()
    r = nqb.TuneResult()
    ds = (ctypes.c_uint * 1)(17)
    assert L.nqb_tune_count(17, ds, 1, None, 64, ctypes.byref(r)) == nqb.E_INVALID      # depth == n
    ds[0] = 5
    assert L.nqb_tune_count(17, ds, 1, None, 0, ctypes.byref(r)) == nqb.E_INVALID       # sample_div 0
    assert L.nqb_tune_count(17, None, 1, None, 64, ctypes.byref(r)) == nqb.E_INVALID
    assert L.nqb_tune_count(3, ds, 1, None, 64, ctypes.byref(r)) == nqb.E_INVALID       # n below 4
    devs = (ctypes.c_int * 1)(0)
    assert L.nqb_solve_states_multi(None, 0, None, 1, None, ctypes.byref(u64), None) == nqb.E_INVALID
    assert L.nqb_solve_states_multi(None, 0, devs, 0, None, ctypes.byref(u64), None) == nqb.E_INVALID
    assert L.nqb_solve_states_multi(None, 5, devs, 1, None, ctypes.byref(u64), None) == nqb.E_INVALID
    for n, d in [(3, 1), (32, 5), (10, 0), (10, 10)]:
        assert L.nqb_generate_pool_device(n, d, ctypes.byref(vp), ctypes.byref(u64), None) == nqb.E_INVALID
    assert L.nqb_measure_int32_peak(0, None, None) == nqb.E_INVALID
    assert L.nqb_trim_device_memory(-1) == nqb.E_NODEVICE
    assert L.nqb_trim_device_memory(64) == nqb.E_NODEVICE
    assert L.nqb_model_predict_ex(None, None, 0, None, 0) == nqb.E_INVALID
    assert L.nqb_device_count(None) == nqb.E_INVALID
    t = nqb.Target()
    assert L.nqb_pool_for_target(8, 0, ctypes.byref(t)) == nqb.E_INVALID
    assert L.nqb_pool_for_target(40, 100, ctypes.byref(t)) == nqb.E_INVALID
    assert L.nqb_pool_for_target(8, 100, None) == nqb.E_INVALID
    ex = L.nqb_batched_launch_ex
    buf = ctypes.create_string_buffer(160)
    base = ctypes.addressof(buf) + (-ctypes.addressof(buf)) % 16  # a 16-byte aligned host address
    out = ctypes.c_uint64(0)
    assert ex(None, 1 << 32, None, base, 64, ctypes.byref(out), None, 0, 0, 0, None) == nqb.E_RANGE
    assert ex(None, 0, None, base, 64, None, None, 0, 0, 0, None) == nqb.E_INVALID          # no result words
    assert ex(None, 0, None, None, 64, ctypes.byref(out), None, 0, 0, 0, None) == nqb.E_INVALID  # no scratch
    assert ex(None, 0, None, base, 2, ctypes.byref(out), None, 0, 0, 0, None) == nqb.E_INVALID   # scratch < head
    assert ex(None, 5, None, base, 64, ctypes.byref(out), None, 0, 0, 0, None) == nqb.E_INVALID  # items missing
    assert ex(None, 0, None, base + 4, 128, ctypes.byref(out), None, 0, 0, 0, None) == nqb.E_INVALID  # ring unaligned
    assert ex(None, 0, None, base, 64, ctypes.byref(out), None, 0, 32, 0, None) == nqb.E_INVALID  # stack depth > 31


def test_c_program_links_and_runs(tmp_path):
    """A C program, as the reference's own code would call the library: compiled against
    include/nqb.h, linked with -lnqb, it sizes a pool by count target, writes it as a state
    file, reads it back and rebuilds the search states (the host-side entry points)."""
    from conftest import PKG_DIR, ROOT
    src = tmp_path / "use_nqb.c"
    src.write_text(r'''
#include <stdio.h>
#include <string.h>
#include "nqb.h"
int main(int argc, char** argv) {
    nqb_target t;
    if (nqb_pool_for_target(10, 1334, &t) != NQB_OK) return 1;
    nqb_placement* pl = NULL; uint64_t cnt = 0;
    if (nqb_generate_pool_placements(10, t.pool_depth, &pl, &cnt) != NQB_OK || cnt != t.count) return 2;
    if (nqb_write_state_file(argv[1], pl, cnt, 10, t.lock_row, 1) != NQB_OK) return 3;
    nqb_state_file info; nqb_placement* back = NULL;
    if (nqb_read_state_file(argv[1], 1, 10, &info, &back) != NQB_OK || info.count != cnt) return 4;
    if (memcmp(pl, back, cnt * sizeof(nqb_placement)) != 0) return 5;
    nqb_state st[700], pool[700]; uint64_t pc = 0;
    if (cnt > 700 || nqb_states_from_placements(back, cnt, 1, st) != NQB_OK) return 6;
    if (nqb_generate_pool_into(10, t.pool_depth, pool, 700, &pc) != NQB_OK || pc != cnt) return 7;
    if (memcmp(st, pool, cnt * sizeof(nqb_state)) != 0) return 8;
    printf("lock %u states %llu\n", t.lock_row, (unsigned long long)cnt);
    nqb_free(pl); nqb_free(back);
    return strcmp(nqb_strerror(NQB_E_FORMAT), "unknown status") == 0 ? 9 : 0;
}
''')
    exe = tmp_path / "use_nqb"
    subprocess.run(["gcc", "-std=c11", "-O1", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", PKG_DIR, "-lnqb", f"-Wl,-rpath,{PKG_DIR}"], check=True)
    p = subprocess.run([str(exe), str(tmp_path / "pool.nqsf")], capture_output=True, text=True)
    assert p.returncode == 0 and p.stdout.strip() == "lock 4 states 697", (p.returncode, p.stdout, p.stderr)
    golden = os.path.join(ROOT, "tests", "golden", "nqsf", "g_n10_1334.nqsf")
    assert (tmp_path / "pool.nqsf").read_bytes() == open(golden, "rb").read()  # the reference CLI's -g 1334


# Entry points that cannot throw: no standard-library container, `new` or thread on their path
# (nqb_count only forwards to nqb_count_ex).
_NO_THROW = {"nqb_version", "nqb_device_count", "nqb_device_check", "nqb_trim_device_memory",
             "nqb_states_from_ref", "nqb_states_from_placements", "nqb_model_get_params",
             "nqb_model_set_params", "nqb_batch_plan_run", "nqb_batch_plan_config", "nqb_debug_fail_allocation",
             "nqb_count"}


def test_entry_points_catch_exceptions(nqb):
    # every entry point returning a status is a function-try-block closed by NQB_ABI_CATCH, so
    # no C++ exception crosses the C ABI (a source check: the body ends in the handler)
    import re
    csrc = os.path.join(os.path.dirname(nqb.__file__), "csrc")
    src = "".join(open(os.path.join(csrc, f)).read() for f in sorted(os.listdir(csrc))
                  if f.endswith((".cu", ".cpp")))
    header = open(os.path.join(os.path.dirname(os.path.dirname(nqb.__file__)), "include", "nqb.h")).read()
    status_fns = set(re.findall(r"^(?:int|long long) (nqb_\w+)\(", header, re.M))
    assert len(status_fns) > 40
    missing = [name for name in sorted(status_fns - _NO_THROW)
               if not re.search(r"^(?:extern \"C\" )?(?:int|long long) " + name +
                                r"\([^{;]*\) try \{\n(?:(?!^\}).*\n)*?\} NQB_ABI_CATCH$", src, re.M)]
    assert not missing, f"not function-try-blocks closed by NQB_ABI_CATCH: {missing}"
