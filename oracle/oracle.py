"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle (oracle/ws_oracle.cpp).

Used by tests/ (as the checker), by __graft_entry__.smoke() and by bench.py's CPU-baseline leg
(as the timed CPU restatement).  Never used by the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libws_oracle.so")

_P = C.c_void_p
_lib = None


def _build_if_missing():
    if not os.path.exists(LIB):
        subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared",
                        "-ffp-contract=off", "-fno-fast-math", os.path.join(HERE, "ws_oracle.cpp"),
                        "-o", LIB], check=True)


def lib():
    global _lib
    if _lib is None:
        _build_if_missing()
        h = C.CDLL(LIB)
        for suf in ("f32", "f64"):
            getattr(h, "ws_oracle_eval_rows_" + suf).argtypes = [
                _P, C.c_int64, C.c_int64, _P, C.c_int64, C.c_int64, _P, C.c_int64, _P, C.c_int,
                _P, _P, _P, C.c_int]
            getattr(h, "ws_oracle_fused_rmse_" + suf).argtypes = [
                _P, C.c_int64, C.c_int64, _P, C.c_int64, C.c_int64, _P, C.c_int64, _P, _P, C.c_int,
                _P, C.c_int]
            getattr(h, "ws_oracle_fitness_" + suf).argtypes = [
                _P, C.c_int64, C.c_int64, _P, C.c_int64, C.c_int64, _P, C.c_int64, _P, _P, C.c_int,
                C.c_int, C.c_int, C.c_double, _P, _P, C.c_int]
        h.ws_oracle_threads.restype = C.c_int
        _lib = h
    return _lib


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else C.c_void_p(0)


def _suffix(dtype):
    return "f32" if np.dtype(dtype) == np.float32 else "f64"


def threads() -> int:
    return lib().ws_oracle_threads()


def eval_rows(tmap, pop, X, consts, strict=0, nthreads=0):
    """K1 semantics: (preds [B, D], sp [B, D] int32, err [B, D] uint8)."""
    pop = np.ascontiguousarray(pop, dtype=np.uint8)
    X = np.ascontiguousarray(X)
    B, L = pop.shape
    V, D = X.shape
    K = consts.shape[1] if consts is not None and consts.ndim == 2 else 0
    c = np.ascontiguousarray(consts, dtype=X.dtype) if K > 0 else None
    preds = np.empty((B, D), dtype=X.dtype)
    sp = np.empty((B, D), dtype=np.int32)
    err = np.empty((B, D), dtype=np.uint8)
    getattr(lib(), "ws_oracle_eval_rows_" + _suffix(X.dtype))(
        _p(pop), B, L, _p(X), V, D, _p(c), K, C.byref(tmap), int(strict), _p(preds), _p(sp),
        _p(err), int(nthreads or threads()))
    return preds, sp, err


def fused_rmse(tmap, pop, X, consts, y, strict=0, nthreads=0):
    """K2 semantics with the reference's exact reduction order: RMSE [B]."""
    pop = np.ascontiguousarray(pop, dtype=np.uint8)
    X = np.ascontiguousarray(X)
    B, L = pop.shape
    V, D = X.shape
    K = consts.shape[1] if consts is not None and consts.ndim == 2 else 0
    c = np.ascontiguousarray(consts, dtype=X.dtype) if K > 0 else None
    y = np.ascontiguousarray(y, dtype=X.dtype)
    out = np.empty(B, dtype=X.dtype)
    getattr(lib(), "ws_oracle_fused_rmse_" + _suffix(X.dtype))(
        _p(pop), B, L, _p(X), V, D, _p(c), K, _p(y), C.byref(tmap), int(strict), _p(out),
        int(nthreads or threads()))
    return out


POLICY = {"fused": 0, "classic": 1}
LOSS = {"rmse": 0, "mse": 1, "r2": 2, "sse": 3}


def fitness(tmap, pop, X, consts, y, strict=0, policy="fused", loss="rmse", invalid_value=None,
            nthreads=0, with_ninv=False):
    """ws_eval_fitness semantics (FP64 sum of T-rounded squares)."""
    pop = np.ascontiguousarray(pop, dtype=np.uint8)
    X = np.ascontiguousarray(X)
    B, L = pop.shape
    V, D = X.shape
    K = consts.shape[1] if consts is not None and consts.ndim == 2 else 0
    c = np.ascontiguousarray(consts, dtype=X.dtype) if K > 0 else None
    y = np.ascontiguousarray(y, dtype=X.dtype)
    if invalid_value is None:
        invalid_value = 1e15 if X.dtype == np.float32 else 1e100
    out = np.empty(B, dtype=np.float64 if loss == "sse" else X.dtype)
    ninv = np.empty(B, dtype=np.int32)
    getattr(lib(), "ws_oracle_fitness_" + _suffix(X.dtype))(
        _p(pop), B, L, _p(X), V, D, _p(c), K, _p(y), C.byref(tmap), int(strict), POLICY[policy],
        LOSS[loss], float(invalid_value), _p(out), _p(ninv), int(nthreads or threads()))
    return (out, ninv) if with_ninv else out
