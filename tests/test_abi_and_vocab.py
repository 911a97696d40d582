"""C ABI surface and bytecode vocabulary (CPU only)."""
import json
import os
import re
import subprocess

import numpy as np
import pytest

import ws_testlib as tl

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.join(tl.REPO, "include", "warpsym.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ws_[a-z0-9_]+)\s*\(", src)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = tl.N.lib()
    syms = declared_symbols()
    assert len(syms) >= 8
    for s in syms:
        assert hasattr(lib, s), s
    nm = subprocess.run(["nm", "-D", "--defined-only", tl.N.LIB_PATH], capture_output=True,
                        text=True, check=True).stdout
    exported = set(re.findall(r"\bT (ws_\w+)", nm))
    assert set(syms) <= exported, set(syms) - exported
    # the ctypes binding declares every entry point of the header
    assert set(tl.N.exported_symbols()) == set(syms)


def test_version_and_workspace_query():
    lib = tl.N.lib()
    assert b"sm_100a" in lib.ws_version()
    b1 = lib.ws_fitness_workspace_bytes(1000, 64, tl.N.WS_F32)
    b2 = lib.ws_fitness_workspace_bytes(2000, 64, tl.N.WS_F32)
    b3 = lib.ws_fitness_workspace_bytes(1000, 64, tl.N.WS_F64)
    assert 0 < b1 < b2 and b1 < b3 and b1 % 256 == 0
    assert lib.ws_schedule_count() >= 1


def test_fused_envelope_errors_match_reference_texts():
    """launch_rpn_eval_fused's checks (rpn_kernels.cu:2539-2545) reject before any GPU work."""
    import ctypes as C
    lib = tl.N.lib()
    g = tl.GPUGrammar(num_variables=5)
    m = tl.token_map(g)
    dummy = C.c_void_p(256)

    def call(B, L, V, D):
        return lib.ws_eval_rpn_fused(0, dummy, B, L, dummy, V, D, dummy, 2, dummy, dummy,
                                     C.byref(m), 0, 0, dummy, 1 << 30, None)

    for args, msg in (((0, 8, 2, 4), "population must be non-empty"),
                      ((4, 8, 5, 4), "fused evaluator supports 1..4 variables"),
                      ((4, 257, 2, 4), "fused evaluator program length exceeds 256"),
                      ((4, 8, 2, 1025), "fused evaluator supports 1..1024 samples")):
        st = call(*args)
        assert st == 1
        assert lib.ws_last_error().decode() == msg


def test_fitness_rejects_bad_arguments_without_gpu():
    import ctypes as C
    lib = tl.N.lib()
    g = tl.GPUGrammar(num_variables=2)
    m = tl.token_map(g)
    opts = tl.N.FitnessOpts(0, 0, 0, 0, 1e15)
    dummy = C.c_void_p(256)
    st = lib.ws_eval_fitness(0, dummy, 4, 300, dummy, 2, 8, None, 0, dummy, dummy, None,
                             C.byref(m), C.byref(opts), dummy, 1 << 30, None)
    assert st == 1 and "program length" in lib.ws_last_error().decode()
    st = lib.ws_eval_fitness(0, dummy, 4, 8, dummy, 2, 8, None, 0, dummy, dummy, None,
                             C.byref(m), C.byref(opts), dummy, 16, None)
    assert st == 3 and "workspace" in lib.ws_last_error().decode()


@pytest.fixture(scope="module")
def vocab():
    with open(os.path.join(HERE, "golden", "vocab_ids.json")) as f:
        return json.load(f)


def test_grammar_ids_match_reference(vocab):
    """Token IDs and the scalar ID argument tuple equal the reference's for each config
    (fixture made by importing the reference's GPUGrammar / CudaRPNVM._cache_ids)."""
    for cfg in vocab:
        g = tl.GPUGrammar(num_variables=cfg["num_variables"], operators=cfg["operators"])
        assert g.token_to_id == cfg["token_to_id"], cfg["name"]
        assert g.vocab_size == cfg["vocab_size"]
        assert list(g.scalar_ids()) == cfg["scalar_ids"], cfg["name"]
        assert g.arities() == cfg["arities"]


def test_token_lut_precedence(vocab):
    """The lookup table follows the reference's precedence: PAD, variables, C, literals,
    binary, unary (rpn_kernels.cu:249-346); unknown IDs map to the error class."""
    import ctypes as C
    lib = tl.N.lib()
    for cfg in vocab:
        g = tl.GPUGrammar(num_variables=cfg["num_variables"], operators=cfg["operators"])
        m = tl.token_map(g)
        cls = np.zeros(256, np.uint8)
        arg = np.zeros(256, np.uint8)
        tl.N.check(lib.ws_debug_token_lut(C.byref(m), len(g.active_variables), 0,
                                          cls.ctypes.data, arg.ctypes.data))
        assert cls[0] == 0
        for i, v in enumerate(g.active_variables):
            t = g.token_to_id[v]
            assert cls[t] == 1 and arg[t] == i
        assert cls[g.token_to_id["C"]] == 2
        for j, lit in enumerate(["0", "1", "2", "3", "4", "5", "6", "10", "pi", "e"]):
            t = g.token_to_id[lit]
            assert cls[t] == 3 and arg[t] == j
        for op in g.operators:
            c = cls[g.token_to_id[op]]
            assert (8 <= c <= 13) if g.token_arity[op] == 2 else (16 <= c <= 32), op
        assert all(cls[t] == 4 for t in range(g.vocab_size, 256))
    # duplicate IDs: the first matching class in the reference's order wins
    g = tl.GPUGrammar(num_variables=2)
    m = tl.token_map(g)
    m.op_sqrt = m.op_sin  # both compare equal: classic order tests sqrt before sin
    cls = np.zeros(256, np.uint8)
    arg = np.zeros(256, np.uint8)
    tl.N.check(lib.ws_debug_token_lut(C.byref(m), 2, 0, cls.ctypes.data, arg.ctypes.data))
    assert cls[m.op_sin] == 21  # T_SQRT
    m.id_C = m.id_x_start  # a variable ID wins over C
    tl.N.check(lib.ws_debug_token_lut(C.byref(m), 2, 0, cls.ctypes.data, arg.ctypes.data))
    assert cls[m.id_x_start] == 1
