"""The bounds-checked build (libnqb_checked.so, NQB_CHECKS): every stack push of the search
kernels is compared with the lane's last slot.  The unchecked kernels rely on the proof
that a search from a state with f free columns never holds more than f - 1 pending rows;
here the same parity cases run with that bound enforced at every step and must come out
exact with no bound flag raised.  Runs in a subprocess, since a process loads one build."""
import json
import os
import subprocess
import sys

import pytest

from conftest import GOLDEN_DIR, ORACLE_DIR, PKG_DIR, ROOT

pytestmark = pytest.mark.gpu
CHECKED = os.path.join(PKG_DIR, "libnqb_checked.so")

SCRIPT = r"""
import json, sys, importlib.util
import numpy as np
spec = importlib.util.spec_from_file_location("nqb", sys.argv[1] + "/__init__.py")
nqb = importlib.util.module_from_spec(spec); spec.loader.exec_module(nqb)
sys.path.insert(0, sys.argv[2]); import nqo
kat = {int(k): v for k, v in json.load(open(sys.argv[3]))["kat_counts"].items()}
out = {"lib": nqb.LIB_PATH, "counts": [], "batch": None}
for n, d in [(8, 1), (10, 9), (12, 11), (13, 3), (15, 4), (16, 5), (17, 5), (18, 6)]:
    for form in (0, 1):
        out["counts"].append([n, d, form, nqb.count(n, d, form=form) == kat[n]])
boards = nqb.sample_boards(nqb.BATCH_SEED, 8192, 16, 20, 3, 7)
got, _ = nqb.solve_batch(boards, form=1)
plain, _ = nqb.solve_batch(boards, form=0)
small = np.flatnonzero((boards["n"] <= 17) & (boards["row"] >= 6))[:100]
want, _ = nqo.solve_states(boards[small])
out["batch"] = bool(np.array_equal(got, plain) and np.array_equal(got[small], want))
print(json.dumps(out))
"""


def test_checked_build_is_exact_with_the_bound_enforced():
    if not os.path.exists(CHECKED):
        pytest.fail(f"{CHECKED} is not built: run `make -C {PKG_DIR} checked`")
    env = dict(os.environ, NQB_LIBRARY=CHECKED)
    p = subprocess.run([sys.executable, "-c", SCRIPT, PKG_DIR, ORACLE_DIR, os.path.join(GOLDEN_DIR, "ref_vectors.json")],
                       capture_output=True, text=True, env=env, timeout=1200, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-3000:]
    r = json.loads(p.stdout.strip().splitlines()[-1])
    assert r["lib"] == CHECKED
    assert all(ok for *_, ok in r["counts"]), r["counts"]
    assert r["batch"]
