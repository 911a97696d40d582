"""Shared helpers of the test-suite: package/oracle loading, program generators for edge
cases, and fitness comparison with the reference's invalid-sentinel classes."""
from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

import __graft_entry__ as _entry  # noqa: E402

pkg = _entry.load_package()
from warpsymbolic_b200 import _native as N  # noqa: E402
from warpsymbolic_b200.grammar import GPUGrammar, PAD_ID, PI_VAL, E_VAL  # noqa: E402
from warpsymbolic_b200 import synthetic  # noqa: E402

_spec = importlib.util.spec_from_file_location("ws_oracle_py", os.path.join(REPO, "oracle", "oracle.py"))
oracle = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(oracle)

# BASELINE config 1 op set: {+, -, *, /, sin, cos, exp, log, sqrt, neg} (pow and abs off).
C1_OPERATORS = ('+', '-', '*', '/', 'sin', 'cos', 'log', 'exp', 'sqrt')
# Every operator the bytecode supports.
ALL_OPERATORS = ('+', '-', '*', '/', 'pow', '%', 'sin', 'cos', 'tan', 'log', 'exp', 'fact',
                 'gamma', 'lgamma', 'asin', 'acos', 'atan', 'floor', 'ceil', 'sign', 'sqrt', 'abs')


def write_report(name: str, obj) -> None:
    """Writes a measurement table as JSON to $WS_REPORT_DIR/<name> when that variable names a
    directory (nothing otherwise)."""
    import json
    out_dir = os.environ.get("WS_REPORT_DIR", "")
    if out_dir and os.path.isdir(out_dir):
        with open(os.path.join(out_dir, name), "w") as f:
            json.dump(obj, f, indent=1)


def token_map(g: GPUGrammar) -> N.TokenMap:
    return N.TokenMap.from_args(*g.scalar_ids(), pi_val=PI_VAL, e_val=E_VAL)


def random_population(g: GPUGrammar, B: int, L: int, K: int, rng, valid_only: bool = True,
                      len_low: int = 1, use_literals: bool = True, const_range=(-2.0, 2.0)):
    """Mixed population: valid programs of random lengths, plus (unless valid_only) token soup
    (underflows, leftovers, unknown IDs), PAD gaps and deep push runs that hit the reference's
    push-drop at depth 32."""
    pop = synthetic.random_programs(g, B, len_low, L, L, rng, max_consts=max(K, 1) + 2,
                                    use_literals=use_literals)
    if not valid_only:
        n_bad = B // 4
        idx = rng.choice(B, size=n_bad, replace=False)
        for j, i in enumerate(idx):
            kind = j % 4
            if kind == 0:  # random token soup (incl. IDs outside the vocabulary)
                n = int(rng.integers(1, L + 1))
                pop[i, :n] = rng.integers(1, 256 if j % 8 == 0 else g.vocab_size, size=n)
                pop[i, n:] = PAD_ID
            elif kind == 1:  # PAD in the middle: tokens after it are ignored
                n = int(rng.integers(1, L))
                pop[i, n] = PAD_ID
            elif kind == 2 and L >= 40:  # 33+ pushes then binaries: push-drop at depth 32
                n_push = int(rng.integers(30, min(L, 40)))
                var_ids = [g.token_to_id[v] for v in g.active_variables] + [g.token_to_id['C']]
                pop[i, :n_push] = rng.choice(var_ids, size=n_push)
                n_bin = min(L - n_push, int(rng.integers(n_push - 3, n_push + 2)))
                bins = [g.token_to_id[o] for o in g.operators if g.token_arity[o] == 2]
                pop[i, n_push:n_push + n_bin] = rng.choice(bins, size=n_bin)
                pop[i, n_push + n_bin:] = PAD_ID
            else:  # drop the last token (usually a leftover or an underflow later)
                row = pop[i]
                n = int(np.argmax(row == PAD_ID)) if (row == PAD_ID).any() else L
                if n > 1:
                    pop[i, n - 1] = PAD_ID
    consts = rng.uniform(*const_range, size=(B, K)).astype(np.float32)
    return pop, consts


def oracle_fitness(g, pop, X, consts, y, policy="classic", loss="rmse", strict=0,
                   invalid_value=None, with_ninv=False):
    return oracle.fitness(token_map(g), pop, X, consts, y, strict=strict, policy=policy,
                          loss=loss, invalid_value=invalid_value, with_ninv=with_ninv)


def classes(v: np.ndarray, iv: float):
    """0 = regular value, 1 = invalid sentinel, 2 = sqrt(sentinel) overflow class."""
    v = np.asarray(v, dtype=np.float64)
    sq = float(np.sqrt(np.float32(iv))) if iv < 1e38 else float(np.sqrt(iv))
    c = np.zeros(v.shape, dtype=np.int8)
    c[np.isclose(v, sq, rtol=1e-5)] = 2
    c[v >= 0.5 * iv] = 1
    return c


def assert_fitness_close(got, ref, rtol=1e-5, atol=1e-6, iv=1e15, min_frac=1.0):
    """Class agreement (invalid / overflow / regular) and closeness of regular values.
    min_frac < 1 tolerates a fraction of mismatches (fast-math GPU vs libm CPU)."""
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    cg, cr = classes(got, iv), classes(ref, iv)
    same_class = cg == cr
    reg = same_class & (cr == 0)
    close = np.ones_like(same_class)
    close[reg] = np.abs(got[reg] - ref[reg]) <= atol + rtol * np.abs(ref[reg])
    ok = same_class & close
    frac = ok.mean() if ok.size else 1.0
    if frac < min_frac:
        bad = np.where(~ok)[0][:10]
        raise AssertionError("fitness mismatch: %.4f%% ok (need %.4f%%); first bad %s: got %s ref %s"
                             % (100 * frac, 100 * min_frac, bad, got[bad], ref[bad]))
    return frac
