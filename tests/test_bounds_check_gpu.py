"""The bounds-checked build on the GPU: small shapes (B <= 64, D in 1..300, L <= 64 with programs
that spill into the global scratch slots) through the fitness pipeline (both schedules' kernels:
D <= 128 several programs per warp, above one row pass per warp; fused and classic policies,
protected and strict operators, FP32 and FP64), the loss-and-gradient kernel (K within and
beyond the register accumulators) and the reference-mode adjoint, run once with libwarpsym.so
and once with libwarpsym_bc.so (tests/bounds_check_run.py in a fresh process each).  Every
output is identical bit for bit and the checked build records no out-of-range index.  No test
provokes an out-of-range access on the GPU; the recording path itself is exercised on the host
(tests/test_bounds_check.py)."""
import os
import subprocess
import sys

import numpy as np
import pytest

import ws_testlib as tl

pytestmark = pytest.mark.gpu
HELPER = os.path.join(os.path.dirname(os.path.abspath(__file__)), "bounds_check_run.py")


def _run(out, lib=None):
    env = dict(os.environ)
    env.pop("WARPSYM_LIB", None)
    if lib:
        env["WARPSYM_LIB"] = lib
    proc = subprocess.run([sys.executable, HELPER, out], env=env, capture_output=True, text=True,
                          timeout=900)
    assert proc.returncode == 0, proc.stderr[-3000:]
    return np.load(out)


def test_checked_build_is_identical_and_records_nothing(tmp_path):
    plain = _run(str(tmp_path / "plain.npz"))
    checked = _run(str(tmp_path / "checked.npz"), tl.N.BC_LIB_PATH)
    assert str(plain["lib"]) == "libwarpsym.so" and str(checked["lib"]) == "libwarpsym_bc.so"
    assert int(plain["bc_enabled"]) == 0 and int(checked["bc_enabled"]) == 1
    assert int(checked["bc_word"]) == 0, hex(int(checked["bc_word"]))
    keys = sorted(k for k in plain.files if not k.startswith("bc_") and k != "lib")
    assert len(keys) == 58 and keys == sorted(k for k in checked.files
                                              if not k.startswith("bc_") and k != "lib")
    for k in keys:
        a, b = plain[k], checked[k]
        assert a.dtype == b.dtype and a.shape == b.shape, k
        ua = a.view(np.uint32 if a.dtype.itemsize == 4 else np.uint64)
        ub = b.view(np.uint32 if b.dtype.itemsize == 4 else np.uint64)
        assert np.array_equal(ua, ub), k
