"""The bounds-checked build (libwarpsym_bc.so, compiled with -DWS_BOUNDS_CHECK) on the CPU: it
exports the same C ABI as libwarpsym.so and reports its checks on; its check records the first
out-of-range index and skips the access (ws_debug_bounds_selftest reads a 4-element host array
at indices 0..5); libwarpsym.so reports the checks off and refuses the self-test.  The device
side runs in tests/test_bounds_check_gpu.py."""
import ctypes as C
import os

import pytest

import ws_testlib as tl

N = tl.N


def _bind(lib):
    lib.ws_bounds_status.restype = C.c_int32
    lib.ws_bounds_status.argtypes = [C.POINTER(C.c_int32), C.POINTER(C.c_uint64), C.c_int32]
    lib.ws_debug_bounds_selftest.restype = C.c_int32
    lib.ws_debug_bounds_selftest.argtypes = [C.POINTER(C.c_uint64)]
    return lib


def _status(lib, reset=0):
    en, w = C.c_int32(-1), C.c_uint64(7)
    assert lib.ws_bounds_status(C.byref(en), C.byref(w), reset) == 0
    return en.value, w.value


@pytest.fixture(scope="module")
def checked():
    assert os.path.exists(N.BC_LIB_PATH), "libwarpsym_bc.so is built by __graft_entry__.build()"
    return _bind(C.CDLL(N.BC_LIB_PATH))


def test_normal_build_has_checks_off():
    lib = _bind(C.CDLL(os.path.join(os.path.dirname(N.BC_LIB_PATH), "libwarpsym.so")))
    assert _status(lib) == (0, 0)
    w = C.c_uint64(5)
    assert lib.ws_debug_bounds_selftest(C.byref(w)) != 0 and w.value == 0


def test_checked_build_exports_the_same_abi(checked):
    for name in N.exported_symbols():
        assert getattr(checked, name) is not None, name


def test_checked_build_records_and_skips(checked):
    assert _status(checked, reset=1)[0] == 1
    assert _status(checked) == (1, 0)
    w = C.c_uint64(0)
    assert checked.ws_debug_bounds_selftest(C.byref(w)) == 0  # the out-of-range reads skipped
    assert w.value == (99 << 32) | 4  # site BC_SELFTEST, the first bad index
    assert _status(checked) == (1, 0)  # the self-test clears its own record
