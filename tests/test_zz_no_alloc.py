"""nqb_batched_launch_static: the batched launch for callers that cannot allocate device
memory (under a framework's caching allocator, or where cudaFree's device-wide
synchronisation is not allowed).  Its queue head lives in the library's own
256-byte device array, so the caller passes only the items and the result words.

Checked through the C ABI against nqb_batched_launch (the entry point that takes a
caller-allocated queue head), on two calls in a row: the array keeps the previous call's
head, so the second call also shows that each call starts from an empty queue.  Counts are
integers and must match exactly.  Kept in a file of its own that pytest collects last."""
import ctypes
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN_DIR

pytestmark = pytest.mark.gpu
KAT = {int(k): v for k, v in json.load(open(os.path.join(GOLDEN_DIR, "ref_vectors.json")))["kat_counts"].items()}


def _static_entry(nqb):
    f = nqb.lib().nqb_batched_launch_static
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_uint,
                  ctypes.c_void_p]
    return f


def test_static_scratch_launch_matches_allocating_launch(nqb):
    torch = pytest.importorskip("torch")
    launch_static = _static_entry(nqb)
    n, d = 16, 5
    pool = nqb.generate_pool(n, d)
    d_items = torch.from_numpy(pool.view(np.uint8).copy()).cuda()
    stream = torch.cuda.current_stream().cuda_stream

    # the existing entry point, with a queue head the caller allocated
    d_head = torch.zeros(1, dtype=torch.int32, device="cuda")
    want = torch.zeros(4, dtype=torch.int64, device="cuda")
    nqb.batched_launch(d_items.data_ptr(), len(pool), d_head.data_ptr(), want.data_ptr(), stack_depth=n - d - 1,
                       stream=stream)

    # two calls in a row of the entry point that allocates nothing
    got = torch.zeros((2, 4), dtype=torch.int64, device="cuda")
    for i in range(2):
        rc = launch_static(d_items.data_ptr(), len(pool), None, got[i].data_ptr(), 0, n - d - 1, stream)
        assert rc == nqb.OK, nqb.strerror(rc)
    torch.cuda.synchronize()

    want = want.cpu().numpy().astype(np.uint64)
    got = got.cpu().numpy().astype(np.uint64)
    assert int(want[0]) == KAT[n] and int(want[3]) == 0
    for i in range(2):
        assert list(got[i]) == list(want), (i, got[i], want)


def test_static_scratch_launch_rejects_too_many_items(nqb):
    launch_static = _static_entry(nqb)
    out = ctypes.c_uint64(0)
    rc = launch_static(ctypes.c_void_p(256), (1 << 31) + 1, None, ctypes.byref(out), 0, 4, None)
    assert rc == nqb.E_RANGE
