"""The C ABI: libnqb.so loads, exports every function include/nqb.h declares, and rejects bad
arguments with status codes (never exiting).  No GPU needed: no compute call is made."""
import ctypes
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
    assert nqb.lib().nqb_version() == 10000
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
