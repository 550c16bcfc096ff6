"""The bounds-checked build, in place of a memory sanitizer: libyamc_b200_checked.so is the
engine compiled with -DYAMC_CHECKED, where every index
the chain kernel computes into its atom, staging, k-entry, scratch, pair-queue, near-atom and
random-window arrays is checked; an index outside its array is recorded (source line) in a
device status word and replaced by 0, so the access stays in bounds, and the call returns
YAMC_EBOUNDS.

* the index check on its own (yamc_bounds_check_selftest, in every build): an in-bounds index
  reads its element and records nothing, an out-of-bounds one (past the end or negative) reads
  element 0 and records a source line;
* the checked library runs chains of the parity tests' small systems (unbiased and force-biased,
  both k-space layouts, one- and two-CTA clusters) through the C ABI with no index out of
  bounds, move for move equal to the oracle, in a child process that loads it (YAMC_LIBRARY).
"""
import ctypes
import os
import subprocess
import sys

import pytest

from yamc_b200 import _lib, build

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _selftest(index, size):
    lib = _lib.load()
    v = ctypes.c_double(0.0)
    line = ctypes.c_int32(-1)
    _lib.check(lib.yamc_bounds_check_selftest(0, index, size, ctypes.byref(v), ctypes.byref(line)),
               "yamc_bounds_check_selftest")
    return v.value, line.value


def test_index_check_records_out_of_bounds():
    assert _selftest(2, 4) == (12.0, 0)
    assert _selftest(0, 1) == (10.0, 0)
    for index, size in ((4, 4), (7, 4), (-1, 4), (1, 1)):
        v, line = _selftest(index, size)
        assert v == 10.0 and line > 0, (index, size, v, line)


def test_normal_build_is_not_checked():
    flag = ctypes.c_int32(-1)
    _lib.check(_lib.load().yamc_checked_build(ctypes.byref(flag)), "yamc_checked_build")
    assert flag.value == 0


CHILD = r'''
import ctypes, sys, tempfile
import numpy as np
sys.path.insert(0, ROOT); sys.path.insert(0, ROOT + "/oracle")
import pyoracle
from yamc_b200 import _lib, api, rng, systems
lib = _lib.load()
flag = ctypes.c_int32(-1)
assert lib.yamc_checked_build(ctypes.byref(flag)) == 0 and flag.value == 1, flag.value
for lam, layout, G in ((0.0, 1, 1), (0.0, 2, 2), (0.1, 2, 1), (0.1, 1, 2)):
    with tempfile.TemporaryDirectory() as d:
        files = systems.write_system(systems.small_spec(xlambda=lam), d, seed=3)
        buf = rng.gfortran_stream(11, 40 * 600 + 10000)
        o = pyoracle.Oracle(files)
        olog, _, ocur = o.run_mc(buf, 600)
        eng = api.Engine.from_files(files)
        eng.set_kspace_layout(layout)
        eng.set_launch(G, 0)
        glog, _, gcur, done, st = eng.run_chain(buf, 600)
        assert st == 0 and done == 600, (lam, layout, G, st, done)
        assert np.array_equal(glog["imol"], olog["imol"]) and np.array_equal(glog["flags"], olog["flags"])
        assert gcur == ocur
        for k in ("du_real", "du_k_coul", "du_k_lj", "du_ext"):
            err = np.abs(glog[k][:400] - olog[k][:400]) / np.maximum(np.abs(olog[k][:400]), 1.0)
            assert err.max() <= 1e-10, (lam, layout, G, k, err.max())
        eng.close()
        o.close()
print("checked chains ok")
'''


def test_checked_library_runs_chains_in_bounds():
    assert os.path.exists(build.LIB_CHECKED), "the bounds-checked library is not built (yamc_b200.build --checked)"
    env = dict(os.environ, YAMC_LIBRARY=build.LIB_CHECKED)
    res = subprocess.run([sys.executable, "-c", f"ROOT = {ROOT!r}\n" + CHILD], env=env, capture_output=True,
                         text=True, timeout=600)
    assert res.returncode == 0 and "checked chains ok" in res.stdout, res.stdout[-2000:] + res.stderr[-4000:]
