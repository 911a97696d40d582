"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle (oracle/ws_oracle.cpp).

Used by tests/ (as the checker), by __graft_entry__.smoke() and by bench.py's CPU-baseline leg
(as the timed CPU restatement).  Never used by the product path.
"""
from __future__ import annotations

import ctypes as C
import glob
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libws_oracle.so")

_P = C.c_void_p
_lib = None


def _build_if_missing():
    srcs = sorted(glob.glob(os.path.join(HERE, "*.cpp")))
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(p) for p in srcs):
        subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared",
                        "-ffp-contract=off", "-fno-fast-math"] + srcs + ["-o", LIB], check=True)


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
        for suf in ("f32", "f64"):
            getattr(h, "ws_oracle_backward_" + suf).argtypes = [
                _P, C.c_int64, C.c_int64, _P, C.c_int64, C.c_int64, _P, C.c_int64, _P, _P, _P,
                _P]
            getattr(h, "ws_oracle_loss_grad_" + suf).argtypes = [
                _P, C.c_int64, C.c_int64, _P, C.c_int64, C.c_int64, _P, C.c_int64, _P, _P, _P,
                _P, _P]
        for suf in ("f32", "f64"):
            getattr(h, "ws_oracle_pso_update_" + suf).argtypes = [
                _P, _P, _P, _P, _P, _P, C.c_float, C.c_float, C.c_float, C.c_int64, C.c_int64,
                C.c_int64]
            getattr(h, "ws_oracle_pso_bests_" + suf).argtypes = [
                _P, _P, _P, _P, _P, _P, C.c_int64, C.c_int64, C.c_int64]
        h.ws_oracle_pso_rmse.argtypes = [_P, C.c_int64, C.c_int64, _P, C.c_int64, C.c_int64, _P,
                                         C.c_int64, _P, _P, _P]
        for suf in ("f32", "f64"):
            getattr(h, "ws_oracle_lbfgs_" + suf).argtypes = [
                _P, C.c_int64, C.c_int64, _P, C.c_int64, _P, C.c_int64, C.c_int64, _P, _P,
                C.c_int, C.c_float, C.c_float, C.c_float, _P]
        h.ws_oracle_simplify.argtypes = [_P, C.c_int64, C.c_int64, _P, C.c_int64, _P, _P, _P,
                                         C.c_int64, C.c_int32, _P]
        for suf in ("f32", "f64"):
            getattr(h, "ws_oracle_gp_step_" + suf).argtypes = [
                _P, C.c_int64, C.c_int64, _P, C.c_int64, _P, _P, _P, _P, C.c_int, _P, C.c_int, _P,
                C.c_int, C.c_uint64, C.c_uint64, C.c_int, C.c_int, C.c_float, C.c_float,
                C.c_float, C.c_float, C.c_float, _P, _P]
        h.ws_oracle_mutate.argtypes = [_P, C.c_int64, _P, _P, _P, C.c_int, _P, C.c_int, _P,
                                       C.c_int, _P, C.c_int, C.c_float, C.c_int]
        h.ws_oracle_splice.argtypes = [_P, _P, C.c_int64, C.c_int64, _P, _P, _P, _P, _P, _P, _P,
                                       C.c_int]
        h.ws_oracle_genrand.argtypes = [_P, C.c_int64, C.c_int, _P, C.c_int, _P, C.c_int, _P,
                                        C.c_int, C.c_uint64, C.c_float, C.c_float, C.c_float]
        h.ws_oracle_batch_best.argtypes = [_P, C.c_int64, C.c_int64, _P, C.c_int64, _P, _P, _P,
                                           _P, _P, C.c_float]
        h.ws_oracle_validate.argtypes = [_P, C.c_int32, C.c_int64, C.c_int64, _P, C.c_int64,
                                         C.c_int32, C.c_int32, _P]
        h.ws_oracle_subtree_ranges.argtypes = [_P, C.c_int64, C.c_int64, _P, C.c_int64,
                                               C.c_int32, _P, _P]
        h.ws_oracle_subtree_length_candidates.argtypes = [_P, C.c_int64, C.c_int64, C.c_int32,
                                                          _P]
        h.ws_oracle_subtree_starts.argtypes = [_P, C.c_int64, C.c_int64, _P, C.c_int64, _P]
        h.ws_oracle_tournament.argtypes = [_P, C.c_int64, _P, C.c_int64, _P, _P, C.c_int64, _P,
                                           _P, _P, C.c_int32, C.c_int32, _P]
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


# ---- the timed CPU baseline -----------------------------------------------------------------
# The same fitness restatement (ws_oracle.cpp) compiled for speed on the host that runs it:
# -O3 -march=native -fopenmp, programs split across all host threads.  It is built where it
# runs (a -march=native binary must not travel to another CPU), into _native/ under a key of the
# host's CPU model and flags.  Timing only: with -O3 the compiler may contract a*b+c into FMAs, so
# the IEEE build above (libws_oracle.so, -O2 -ffp-contract=off) stays the checker.
NATIVE_FLAGS = ["-O3", "-march=native", "-fopenmp"]
_timed = None


def _host_key() -> str:
    import hashlib
    info = ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith(("model name", "flags")):
                    info += line
                    if line.startswith("flags"):
                        break
    except OSError:
        pass
    return hashlib.sha1(info.encode()).hexdigest()[:12]


def timed_lib_path() -> str:
    return os.path.join(HERE, "_native", "libws_oracle_native_%s.so" % _host_key())


def timed_lib():
    """ctypes handle of the host-tuned fitness restatement (built on first use)."""
    global _timed
    if _timed is None:
        path = timed_lib_path()
        src = os.path.join(HERE, "ws_oracle.cpp")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            os.makedirs(os.path.dirname(path), exist_ok=True)
            tmp = path + ".tmp%d" % os.getpid()
            subprocess.run(["g++", "-std=c++17", "-fPIC", "-shared"] + NATIVE_FLAGS +
                           [src, "-o", tmp], check=True)
            os.replace(tmp, path)
        h = C.CDLL(path)
        for suf in ("f32", "f64"):
            getattr(h, "ws_oracle_fitness_" + suf).argtypes = [
                _P, C.c_int64, C.c_int64, _P, C.c_int64, C.c_int64, _P, C.c_int64, _P, _P, C.c_int,
                C.c_int, C.c_int, C.c_double, _P, _P, C.c_int]
        h.ws_oracle_threads.restype = C.c_int
        _timed = h
    return _timed


def fitness(tmap, pop, X, consts, y, strict=0, policy="fused", loss="rmse", invalid_value=None,
            nthreads=0, with_ninv=False, timed=False):
    """ws_eval_fitness semantics (FP64 sum of T-rounded squares).  timed=True runs the
    host-tuned build (the timed CPU baseline) instead of the IEEE checker."""
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
    h = timed_lib() if timed else lib()
    getattr(h, "ws_oracle_fitness_" + _suffix(X.dtype))(
        _p(pop), B, L, _p(X), V, D, _p(c), K, _p(y), C.byref(tmap), int(strict), POLICY[policy],
        LOSS[loss], float(invalid_value), _p(out), _p(ninv), int(nthreads or h.ws_oracle_threads()))
    return (out, ninv) if with_ninv else out


def backward(tmap, pop, X, consts, gout):
    """eval_rpn_backward semantics: (grad [B, K] float64, sum of |terms| [B, K])."""
    pop = np.ascontiguousarray(pop, dtype=np.uint8)
    X = np.ascontiguousarray(X)
    B, L = pop.shape
    V, D = X.shape
    c = np.ascontiguousarray(consts, dtype=X.dtype)
    K = c.shape[1]
    g = np.ascontiguousarray(gout, dtype=X.dtype).reshape(B, D)
    grad = np.empty((B, K), dtype=np.float64)
    absg = np.empty((B, K), dtype=np.float64)
    getattr(lib(), "ws_oracle_backward_" + _suffix(X.dtype))(
        _p(pop), B, L, _p(X), V, D, _p(c), K, _p(g), C.byref(tmap), _p(grad), _p(absg))
    return grad, absg


def loss_grad(tmap, pop, X, consts, y):
    """Loss mode of the adjoint restatement: (loss [B] float64 = mean_d (pred - y)^2, infinite
    without a result; grad [B, K] float64 = d loss / d C; sum of |terms| [B, K])."""
    pop = np.ascontiguousarray(pop, dtype=np.uint8)
    X = np.ascontiguousarray(X)
    B, L = pop.shape
    V, D = X.shape
    c = np.ascontiguousarray(consts, dtype=X.dtype).reshape(B, -1)
    K = c.shape[1]
    yy = np.ascontiguousarray(y, dtype=X.dtype).reshape(D)
    loss = np.empty(B, dtype=np.float64)
    grad = np.empty((B, K), dtype=np.float64)
    absg = np.empty((B, K), dtype=np.float64)
    getattr(lib(), "ws_oracle_loss_grad_" + _suffix(X.dtype))(
        _p(pop), B, L, _p(X), V, D, _p(c), K, _p(yy), C.byref(tmap), _p(loss), _p(grad),
        _p(absg))
    return loss, grad, absg


# ---------------------------------------------------------------------------------------------
# Population structure (oracle/ws_oracle_structure.cpp).

VALIDATE_MODES = {"kernel": 0, "clamped": 1, "stack": 2}


def validate(pop, arities, pad_id=0, mode="kernel"):
    """bool [B] under the reference rule `mode` (kernel / clamped / stack)."""
    pop = np.ascontiguousarray(pop)
    assert pop.dtype in (np.uint8, np.int64)
    ar = np.ascontiguousarray(arities, dtype=np.int32)
    B, L = pop.shape
    out = np.empty(B, dtype=np.uint8)
    lib().ws_oracle_validate(_p(pop), pop.itemsize, B, L, _p(ar), ar.size, int(pad_id),
                             VALIDATE_MODES[mode], _p(out))
    return out.astype(bool)


def subtree_ranges(pop, arities, pad_id=0):
    """(starts int64 [B, L], lengths int64 [B]) by find_subtree_ranges_kernel's backward scan."""
    pop = np.ascontiguousarray(pop, dtype=np.uint8)
    ar = np.ascontiguousarray(arities, dtype=np.int32)
    B, L = pop.shape
    starts = np.empty((B, L), dtype=np.int64)
    lengths = np.empty(B, dtype=np.int64)
    lib().ws_oracle_subtree_ranges(_p(pop), B, L, _p(ar), ar.size, int(pad_id), _p(starts),
                                   _p(lengths))
    return starts, lengths


def subtree_length_candidates(pop, pad_id=0):
    """bool [B, L+1]: the values the reference's racing out_lengths stores may leave."""
    pop = np.ascontiguousarray(pop, dtype=np.uint8)
    B, L = pop.shape
    cand = np.empty((B, L + 1), dtype=np.uint8)
    lib().ws_oracle_subtree_length_candidates(_p(pop), B, L, int(pad_id), _p(cand))
    return cand.astype(bool)


def subtree_starts(pop, arities):
    """int64 [B, L] by precompute_subtree_starts_kernel's forward recurrence."""
    pop = np.ascontiguousarray(pop, dtype=np.int64)
    ar = np.ascontiguousarray(arities, dtype=np.int32)
    B, L = pop.shape
    out = np.empty((B, L), dtype=np.int64)
    lib().ws_oracle_subtree_starts(_p(pop), B, L, _p(ar), ar.size, _p(out))
    return out


def tournament(fitness, cand, errors=None, cases=None, lengths=None, mad_eps=None,
               island_size=0, n_islands=1):
    """int64 [B] winners; cand int64 [B, T] indices, or int32 [B, T] island offsets."""
    fit = np.ascontiguousarray(fitness, dtype=np.float32)
    cand = np.ascontiguousarray(cand)
    B, T = cand.shape
    f32 = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
    errors, lengths, mad_eps = f32(errors), f32(lengths), f32(mad_eps)
    cases = None if cases is None else np.ascontiguousarray(cases, dtype=np.int32)
    n_data = errors.shape[1] if errors is not None else 0
    out = np.empty(B, dtype=np.int64)
    idx = cand if cand.dtype == np.int64 else None
    off = cand if cand.dtype == np.int32 else None
    assert idx is not None or off is not None
    lib().ws_oracle_tournament(_p(fit), B, _p(errors), n_data, _p(idx), _p(off), T, _p(cases),
                               _p(lengths), _p(mad_eps), int(island_size), int(n_islands), _p(out))
    return out


# ---------------------------------------------------------------------------------------------
# Particle swarm (oracle/ws_oracle_pso.cpp).

def pso_update(pos, vel, pbest, gbest, r1, r2, w, c1, c2):
    """Returns updated (pos, vel) copies; arrays [B, P, K], gbest [B, K]."""
    pos, vel = np.array(pos, copy=True, order="C"), np.array(vel, copy=True, order="C")
    B, P, K = pos.shape
    arr = [np.ascontiguousarray(a, dtype=pos.dtype) for a in (pbest, gbest, r1, r2)]
    getattr(lib(), "ws_oracle_pso_update_" + _suffix(pos.dtype))(
        _p(pos), _p(vel), *[_p(a) for a in arr], float(w), float(c1), float(c2), B, P, K)
    return pos, vel


def pso_update_bests(cur_err, pb_err, pb_pos, cur_pos, gb_err, gb_pos):
    """Returns updated (pb_err, pb_pos, gb_err, gb_pos) copies."""
    out = [np.array(a, copy=True, order="C") for a in (pb_err, pb_pos, gb_err, gb_pos)]
    ce = np.ascontiguousarray(cur_err, dtype=out[0].dtype)
    cp = np.ascontiguousarray(cur_pos, dtype=out[0].dtype)
    B, P = out[0].shape
    K = out[1].shape[2]
    getattr(lib(), "ws_oracle_pso_bests_" + _suffix(out[0].dtype))(
        _p(ce), _p(out[0]), _p(out[1]), _p(cp), _p(out[2]), _p(out[3]), B, P, K)
    return tuple(out)


def pso_rmse(tmap, pop, X, consts, y):
    """RMSE [B] under the fused PSO's evaluator (float32; 1e30 when a row fails)."""
    pop = np.ascontiguousarray(pop, dtype=np.uint8)
    X = np.ascontiguousarray(X, dtype=np.float32)
    c = np.ascontiguousarray(consts, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.float32)
    B, L = pop.shape
    V, D = X.shape
    out = np.empty(B, dtype=np.float32)
    lib().ws_oracle_pso_rmse(_p(pop), B, L, _p(X), V, D, _p(c), c.shape[1], _p(y),
                             C.byref(tmap), _p(out))
    return out


# ---------------------------------------------------------------------------------------------
# L-BFGS kernel semantics (oracle/ws_oracle_lbfgs.cpp).

def lbfgs(tmap, pop, X, consts, y, max_iter=20, gtol=1e-7, cmin=-25.0, cmax=25.0):
    """Returns (constants [B, K] after fitting, rmse [B])."""
    pop = np.ascontiguousarray(pop, dtype=np.uint8)
    X = np.ascontiguousarray(X)
    c = np.array(consts, dtype=X.dtype, copy=True, order="C")
    y = np.ascontiguousarray(y, dtype=X.dtype)
    B, L = pop.shape
    V, D = X.shape
    out = np.empty(B, dtype=X.dtype)
    getattr(lib(), "ws_oracle_lbfgs_" + _suffix(X.dtype))(
        _p(pop), B, L, _p(c), c.shape[1], _p(X), V, D, _p(y), _p(out), int(max_iter),
        float(gtol), float(cmin), float(cmax), C.byref(tmap))
    return c, out


# ---------------------------------------------------------------------------------------------
# Simplifier (oracle/ws_oracle_simplify.cpp).

def simplify(pop, arities, val_table, lit_ids, lit_vals, max_passes, ids29):
    """Returns the simplified copy of int64 pop [B, L]; ids29: the 29 operator / literal IDs in
    the kernel's argument order."""
    out = np.array(pop, dtype=np.int64, copy=True, order="C")
    ar = np.ascontiguousarray(arities, dtype=np.int32)
    vt = np.ascontiguousarray(val_table, dtype=np.float32)
    li = np.ascontiguousarray(lit_ids, dtype=np.int64)
    lv = np.ascontiguousarray(lit_vals, dtype=np.float32)
    idv = np.ascontiguousarray(ids29, dtype=np.int32)
    assert idv.size == 29
    B, L = out.shape
    lib().ws_oracle_simplify(_p(out), B, L, _p(ar), ar.size, _p(vt), _p(li), _p(lv), li.size,
                             int(max_passes), _p(idv))
    return out


def gp_tables(grammar):
    """(arity[256], kind[256], variables, unary ops, binary ops) of a GPUGrammar, as the GP step
    classifies tokens: arity 0 leaf / 1 unary / 2 binary / 3 PAD / 4 other; kind 1 variable,
    2 C, 3 operator, 4 literal, 0 other; the lists in ascending token ID."""
    arity = np.full(256, 4, dtype=np.uint8)
    kind = np.zeros(256, dtype=np.uint8)
    arity[0] = 3
    for tok, i in grammar.token_to_id.items():
        if i == 0:
            continue
        a = grammar.token_arity.get(tok, 0)
        arity[i] = a
        if tok in grammar.active_variables:
            kind[i] = 1
        elif tok == "C":
            kind[i] = 2
        elif a == 0:
            kind[i] = 4
        else:
            kind[i] = 3
    ids = np.arange(256)
    vars_ = ids[kind == 1].astype(np.uint8)
    uns = ids[(kind == 3) & (arity == 1)].astype(np.uint8)
    bins = ids[(kind == 3) & (arity == 2)].astype(np.uint8)
    return arity, kind, vars_, uns, bins


def gp_step(grammar, pop, consts, fitness, seed, generation, tournament_size=3, elitism=1,
            crossover_rate=0.7, mutation_rate=0.05, const_mutation_rate=0.1, const_sigma=0.1,
            parsimony_eps=1e-9):
    """One generation of the B200 GP step on the CPU: (next population, next constants)."""
    pop = np.ascontiguousarray(pop, dtype=np.uint8)
    B, L = pop.shape
    dt = np.float64 if consts.dtype == np.float64 else np.float32
    consts = np.ascontiguousarray(consts, dtype=dt)
    fitness = np.ascontiguousarray(fitness, dtype=dt)
    K = consts.shape[1]
    arity, kind, vars_, uns, bins = gp_tables(grammar)
    out_p = np.zeros_like(pop)
    out_c = np.zeros_like(consts)
    getattr(lib(), "ws_oracle_gp_step_" + _suffix(dt))(
        _p(pop), B, L, _p(consts), K, _p(fitness), _p(arity), _p(kind), _p(vars_), len(vars_),
        _p(uns), len(uns), _p(bins), len(bins), seed, generation, tournament_size, elitism,
        crossover_rate, mutation_rate, const_mutation_rate, const_sigma, parsimony_eps,
        _p(out_p), _p(out_c))
    return out_p, out_c


def mutate(pop, rand_floats, rand_ints, arities, a0, a1, a2, rate, pad=0):
    out = np.ascontiguousarray(pop, dtype=np.uint8).copy()
    rf = np.ascontiguousarray(rand_floats, dtype=np.float32)
    ri = np.ascontiguousarray(rand_ints, dtype=np.int64)
    ar = np.ascontiguousarray(arities, dtype=np.int32)
    a0, a1, a2 = (np.ascontiguousarray(a, dtype=np.uint8) for a in (a0, a1, a2))
    lib().ws_oracle_mutate(_p(out), out.size, _p(rf), _p(ri), _p(ar), len(ar), _p(a0), len(a0),
                           _p(a1), len(a1), _p(a2), len(a2), rate, pad)
    return out


def splice(p1, p2, s1, e1, s2, e2, mask=None, pad=0):
    p1 = np.ascontiguousarray(p1, dtype=np.uint8)
    p2 = np.ascontiguousarray(p2, dtype=np.uint8)
    N, L = p1.shape
    ss = [np.ascontiguousarray(a, dtype=np.int64) for a in (s1, e1, s2, e2)]
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    c1, c2 = np.zeros_like(p1), np.zeros_like(p2)
    lib().ws_oracle_splice(_p(p1), _p(p2), N, L, *[_p(a) for a in ss], _p(m) if m is not None else None,
                           _p(c1), _p(c2), pad)
    return c1, c2


def genrand(B, L, term, un, binr, seed, wt, wu, wb):
    term, un, binr = (np.ascontiguousarray(a, dtype=np.uint8) for a in (term, un, binr))
    out = np.zeros((B, L), dtype=np.uint8)
    lib().ws_oracle_genrand(_p(out), B, L, _p(term), len(term), _p(un), len(un), _p(binr),
                            len(binr), seed, wt, wu, wb)
    return out


def batch_best(pop, consts, fit, best_rmse, tol=1e-9):
    """(best_rpn [L], best_consts [K], best_rmse, best_idx) after one single-block update from
    an empty tracker with `best_rmse`."""
    pop = np.ascontiguousarray(pop, dtype=np.uint8)
    consts = np.ascontiguousarray(consts, dtype=np.float32)
    fit = np.ascontiguousarray(fit, dtype=np.float32)
    B, L = pop.shape
    K = consts.shape[1]
    rpn = np.zeros(L, np.uint8)
    bc = np.zeros(max(K, 1), np.float32)
    br = np.array([best_rmse], np.float32)
    bi = np.array([-1], np.int32)
    lib().ws_oracle_batch_best(_p(pop), B, L, _p(consts), K, _p(fit), _p(rpn), _p(bc), _p(br),
                               _p(bi), tol)
    return rpn, bc[:K], float(br[0]), int(bi[0])
