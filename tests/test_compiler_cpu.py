"""Exact CPU verification of the program compiler (tape) against the oracle (CPU only).

ws_debug_compile + ws_debug_run_tape run the evaluator's compiler and a scalar interpreter of
its tape on the host with the C library's math.  For every (program, row) the oracle's direct
stack interpretation (a restatement of rpn_eval_kernel, rpn_kernels.cu:202-358) must give the
same validity and, for valid rows, the bit-identical value.  This covers constant folding,
Sethi-Ullman reordering, spill slots, push-drop at depth 32, constant-slot clamping, PAD gaps,
unknown tokens and strict-mode errors.
"""
import ctypes as C

import numpy as np
import pytest

import ws_testlib as tl


def compile_host(g, prog, consts, strict, dtype=np.float32):
    lib = tl.N.lib()
    m = tl.token_map(g)
    L = len(prog)
    cap = max(L, 1)  # one tape word per operator
    ctrl = np.zeros(cap, np.uint32)
    imm = np.zeros(cap, np.float64)
    hdr = np.zeros(4, np.int32)
    prog = np.ascontiguousarray(prog, np.uint8)
    c = np.ascontiguousarray(consts, dtype)
    code = tl.N.WS_F32 if dtype == np.float32 else tl.N.WS_F64
    tl.N.check(lib.ws_debug_compile(code, prog.ctypes.data, L, c.ctypes.data if c.size else None,
                                    c.size, C.byref(m), len(g.active_variables), strict, 0,
                                    ctrl.ctypes.data, imm.ctypes.data, hdr.ctypes.data))
    return ctrl, imm, hdr


def run_host(ctrl, imm, n, X, strict):
    lib = tl.N.lib()
    D = X.shape[1]
    pred = np.zeros(D, X.dtype)
    err = np.zeros(D, np.uint8)
    code = tl.N.WS_F32 if X.dtype == np.float32 else tl.N.WS_F64
    Xc = np.ascontiguousarray(X)
    tl.N.check(lib.ws_debug_run_tape(code, ctrl.ctypes.data, imm.ctypes.data, n, Xc.ctypes.data,
                                     D, strict, pred.ctypes.data, err.ctypes.data))
    return pred, err


def spill_bound(L):
    n = (L + 1) // 3
    return int(np.floor(np.log2(n))) if n >= 1 else 0


def check_population(g, pop, consts, X, strict, dtype):
    X = X.astype(dtype)
    consts = consts.astype(dtype)
    preds, sp, err = tl.oracle.eval_rows(tl.token_map(g), pop, X, consts, strict=strict)
    ref_valid = (sp == 1) & (err == 0) & np.isfinite(preds)
    n_checked = 0
    for b in range(pop.shape[0]):
        ctrl, imm, hdr = compile_host(g, pop[b], consts[b], strict, dtype)
        n_instr, status, slots, ntok = hdr
        if status != 0:
            # statically invalid: the reference must fail on every row
            assert not ref_valid[b].any(), (b, pop[b])
            continue
        assert slots <= spill_bound(pop.shape[1]), (slots, pop[b])
        pred, e = run_host(ctrl, imm, int(n_instr), X, strict)
        valid = (e == 0) & np.isfinite(pred)
        assert np.array_equal(valid, ref_valid[b]), (b, pop[b], valid, ref_valid[b])
        vv = ref_valid[b]
        assert np.array_equal(pred[vv].view(np.uint32 if dtype == np.float32 else np.uint64),
                              preds[b][vv].view(np.uint32 if dtype == np.float32 else np.uint64)), \
            (b, pop[b], pred[vv][:4], preds[b][vv][:4])
        n_checked += 1
    return n_checked


@pytest.mark.parametrize("strict", [0, 1])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_compiled_tape_matches_stack_interpreter(strict, dtype):
    rng = np.random.default_rng(1234 + strict)
    g = tl.GPUGrammar(num_variables=3, operators=tl.ALL_OPERATORS)
    pop, consts = tl.random_population(g, 600, 48, 6, rng, valid_only=False)
    X = rng.uniform(-3, 3, size=(3, 37))
    X[:, :3] = [[0.0, -1.0, 1e-10], [2.0, 0.0, -0.0], [1.0, 3.0, -2.5]]  # domain edges
    n = check_population(g, pop, consts, X, strict, dtype)
    assert n > 300


def test_deep_programs_and_push_drop():
    """Long programs (L=256) with deep stacks, balanced trees needing the most spill slots, and
    push runs beyond depth 32 whose extra pushes the reference drops."""
    rng = np.random.default_rng(7)
    g = tl.GPUGrammar(num_variables=2, operators=tl.C1_OPERATORS)
    L = 256
    rows = []
    x0, x1, c = g.token_to_id["x0"], g.token_to_id["x1"], g.token_to_id["C"]
    add, mul, sub = g.token_to_id["+"], g.token_to_id["*"], g.token_to_id["-"]
    sin = g.token_to_id["sin"]

    def balanced(depth):
        if depth == 0:
            return [x0 if rng.random() < 0.5 else x1, sin]
        return balanced(depth - 1) + balanced(depth - 1) + [[add, mul, sub][int(rng.integers(3))]]

    for d in range(1, 7):
        t = balanced(d)
        if len(t) <= L:
            rows.append(t)
    rows.append([x0] * 40 + [add] * 31)          # 40 pushes: 8 dropped, result valid
    rows.append([x0] * 33 + [add] * 31)          # 33 pushes: 1 dropped, valid
    rows.append([x0] * 33 + [add] * 32)          # underflow after the drop
    rows.append([c] * 36 + [add] * 31)           # C slots consumed by dropped pushes
    pop = np.zeros((len(rows), L), np.uint8)
    for i, r in enumerate(rows):
        pop[i, :len(r)] = r
    consts = rng.uniform(-2, 2, size=(len(rows), 40)).astype(np.float32)
    X = rng.uniform(-3, 3, size=(2, 19))
    n = check_population(g, pop, consts, X, 0, np.float32)
    assert n == len(rows) - 1
    ctrl, imm, hdr = compile_host(g, pop[5], consts[5], 0)
    assert hdr[2] == 6  # the depth-6 balanced tree of unary units needs 6 spill slots


def test_constant_only_program_folds_to_one_instruction():
    g = tl.GPUGrammar(num_variables=1)
    prog = g.encode(["C", "2", "*", "sin", "pi", "+"], 8)
    ctrl, imm, hdr = compile_host(g, np.array(prog), np.array([0.7], np.float32), 0)
    assert hdr[0] == 1 and hdr[1] == 0 and hdr[3] == 6
    expected = np.sin(np.float32(0.7) * np.float32(2.0)) + np.float32(3.14159265359)
    assert np.float32(imm[0]) == np.float32(expected)


def test_fold_error_makes_program_invalid_in_strict_mode():
    g = tl.GPUGrammar(num_variables=1)
    prog = g.encode(["0", "log", "x0", "+"], 6)  # log(0) is a strict-mode domain error
    ctrl, imm, hdr = compile_host(g, np.array(prog), np.zeros(0, np.float32), 1)
    assert hdr[1] == 1
    ctrl, imm, hdr = compile_host(g, np.array(prog), np.zeros(0, np.float32), 0)
    assert hdr[1] == 0


def _deep_trees(g, n, rng, L):
    names = g.active_variables + ['C', '1', 'pi']
    bins = [o for o in g.operators if g.token_arity[o] == 2]
    uns = [o for o in g.operators if g.token_arity[o] == 1]
    pop = np.zeros((n, L), dtype=np.uint8)
    for i in range(n):
        def build(depth):
            if depth == 0:
                return [names[int(rng.integers(len(names)))]]
            t = build(depth - 1) + build(depth - 1) + [bins[int(rng.integers(len(bins)))]]
            if uns and rng.random() < 0.3:
                t.append(uns[int(rng.integers(len(uns)))])
            return t
        toks = build(int(rng.integers(1, 6)))[:L]
        pop[i, :len(toks)] = [g.token_to_id[t] for t in toks]
    return pop


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("strict", [0, 1])
@pytest.mark.parametrize("L,xmul", [(30, 1), (64, 7), (64, 100), (200, 2)])
def test_linear_emitter_matches_depth_first(dtype, strict, L, xmul):
    """The device compiler's linear emitter writes the depth-first emitter's tape word for word:
    headers (status, length, spill slots, tokens) and every (ctrl, immediate) pair, over random
    valid programs, token soup with invalid rows, PAD gaps and push-drop runs, literal-rich
    (constant-folded) programs, complete trees that use the deepest spill slots, every operator,
    and offsets that do not fit the tape word."""
    rng = np.random.default_rng(L * 10 + xmul + 3 * strict)
    g = tl.GPUGrammar(num_variables=4, operators=tl.ALL_OPERATORS)
    parts = [tl.random_population(g, 3000, L, 6, rng, valid_only=False)[0],
             tl.random_population(g, 1000, L, 6, rng, valid_only=True, use_literals=True)[0],
             _deep_trees(g, 500, rng, L)]
    pop = np.ascontiguousarray(np.concatenate(parts))
    for K in (0, 1, 6):
        consts = np.ascontiguousarray(rng.uniform(-3, 3, size=(len(pop), max(K, 1)))
                                      .astype(dtype)[:, :K])
        bad = C.c_int64(-1)
        code = tl.N.WS_F32 if dtype == np.float32 else tl.N.WS_F64
        tl.N.check(tl.N.lib().ws_debug_compile_agree(
            code, pop.ctypes.data, len(pop), L, consts.ctypes.data if K else None, K,
            C.byref(tl.token_map(g)), len(g.active_variables), strict, 0, xmul, C.byref(bad)))
        assert bad.value == 0, (K, bad.value)
