"""Generates tests/golden/vocab_ids.json and tests/golden/kats.json.

vocab_ids.json is produced by importing the REFERENCE's own Python modules (GPUGrammar from
src/warpsymbolic/gpu/grammar.py and CudaRPNVM._cache_ids from src/warpsymbolic/gpu/cuda_vm.py)
for several operator configurations; it pins the bytecode (token IDs) and the ~36 scalar ID
arguments every evaluator entry point receives.  Needs the reference checkout, named by
WS_REFERENCE_ROOT; the GPU is not needed.

kats.json transcribes the known-answer tests of the reference test-suite for this path, with
the file:line each comes from.

Usage: WS_REFERENCE_ROOT=<checkout> python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("WS_REFERENCE_ROOT") or sys.exit("set WS_REFERENCE_ROOT to the reference checkout")

ALL_FLAGS = ["PLUS", "MINUS", "MULT", "DIV", "POW", "MOD", "SIN", "COS", "TAN", "LOG", "EXP",
             "FACT", "GAMMA", "LGAMMA", "ASIN", "ACOS", "ATAN", "FLOOR", "CEIL", "SIGN", "SQRT",
             "ABS"]
FLAG_OF = {'+': "PLUS", '-': "MINUS", '*': "MULT", '/': "DIV", 'pow': "POW", '%': "MOD",
           'sin': "SIN", 'cos': "COS", 'tan': "TAN", 'log': "LOG", 'exp': "EXP", 'fact': "FACT",
           'gamma': "GAMMA", 'lgamma': "LGAMMA", 'asin': "ASIN", 'acos': "ACOS", 'atan': "ATAN",
           'floor': "FLOOR", 'ceil': "CEIL", 'sign': "SIGN", 'sqrt': "SQRT", 'abs': "ABS"}

CONFIGS = [
    {"name": "default_1var", "num_variables": 1, "operators": None},
    {"name": "bench_c1_2var", "num_variables": 2,
     "operators": ['+', '-', '*', '/', 'sin', 'cos', 'log', 'exp', 'sqrt']},
    {"name": "bench_c2_5var", "num_variables": 5,
     "operators": ['+', '-', '*', '/', 'sin', 'cos', 'log', 'exp', 'sqrt']},
    {"name": "all_ops_3var", "num_variables": 3, "operators": list(FLAG_OF)},
    {"name": "default_4var", "num_variables": 4, "operators": None},
    {"name": "arith_10var", "num_variables": 10, "operators": ['+', '-', '*', '/']},
]


def vocab_fixture():
    sys.path.insert(0, os.path.join(REF, "src"))
    from warpsymbolic.gpu.config import GpuGlobals
    from warpsymbolic.gpu.grammar import GPUGrammar
    from warpsymbolic.gpu.cuda_vm import CudaRPNVM

    saved = {f: getattr(GpuGlobals, "USE_OP_" + f) for f in ALL_FLAGS}
    out = []
    try:
        for cfg in CONFIGS:
            if cfg["operators"] is not None:
                on = {FLAG_OF[o] for o in cfg["operators"]}
                for f in ALL_FLAGS:
                    setattr(GpuGlobals, "USE_OP_" + f, f in on)
            else:
                for f, v in saved.items():
                    setattr(GpuGlobals, "USE_OP_" + f, v)
            g = GPUGrammar(num_variables=cfg["num_variables"])
            vm = CudaRPNVM.__new__(CudaRPNVM)
            vm.grammar = g
            vm._cache_ids()
            ids = [vm.PAD_ID, vm.id_x_start, vm.id_C, vm.id_pi, vm.id_e, vm.id_0, vm.id_1,
                   vm.id_2, vm.id_3, vm.id_4, vm.id_5, vm.id_6, vm.id_10, vm.op_add, vm.op_sub,
                   vm.op_mul, vm.op_div, vm.op_pow, vm.op_mod, vm.op_sin, vm.op_cos, vm.op_tan,
                   vm.op_log, vm.op_exp, vm.op_sqrt, vm.op_abs, vm.op_neg, vm.op_fact,
                   vm.op_floor, vm.op_ceil, vm.op_sign, vm.op_gamma, vm.op_lgamma, vm.op_asin,
                   vm.op_acos, vm.op_atan]
            out.append({"name": cfg["name"], "num_variables": cfg["num_variables"],
                        "operators": cfg["operators"], "token_to_id": g.token_to_id,
                        "vocab_size": g.vocab_size, "scalar_ids": ids,
                        "arities": [int(a) for a in g.get_arity_tensor().tolist()]})
    finally:
        for f, v in saved.items():
            setattr(GpuGlobals, "USE_OP_" + f, v)
    return out


KATS = {
    "rmse_sqrt_7_5": {
        "source": "tests/gpu/test_new_bugs_v3.py:461-490",
        "grammar": {"num_variables": 1, "operators": None},
        "program": ["x0"], "L": 10, "K": 5, "constants": [0.0] * 5,
        "x": [[1.0, 2.0, 3.0, 4.0]], "y": [2.0, 4.0, 6.0, 8.0], "dtype": "float64",
        "expected_rmse": 2.7386127875258306, "places": 3,
    },
    "x4_passthrough": {
        "source": "tests/gpu/test_cuda_eval_modes.py:137-160",
        "grammar": {"num_variables": 5, "operators": None},
        "program": ["x4"], "L": 64, "K": 0, "rows": 41, "y_is_x": 4, "dtype": "float32",
        "expected_rmse": 0.0, "atol": 1e-7,
    },
    "mode_agreement_programs": {
        "source": "tests/gpu/test_cuda_eval_modes.py:51-132",
        "grammar": {"num_variables": 1, "operators": None},
        "programs": [["x0"], ["x0", "x0", "*"], ["C", "x0", "+"], ["x0", "log"], ["x0", "exp"]],
        "x_linspace": [-2.0, 100.0], "samples": [1, 17, 32, 33, 200, 1024], "y": "zeros",
        "rtol": 2e-5, "atol": 2e-5, "rtol_f64": 1e-10, "invalid_threshold": 1e14,
    },
    "validator_rejects_prefix_underflow": {
        "source": "tests/gpu/test_gpu_rpn_validation_regressions.py:14-46",
        "grammar": {"num_variables": 1, "operators": None},
        "programs": [["+", "x0", "x0"], ["sin", "x0"]], "L": 4, "expected_valid": [False, False],
    },
}


def main():
    vocab = vocab_fixture()
    with open(os.path.join(HERE, "vocab_ids.json"), "w") as f:
        json.dump(vocab, f, indent=1, sort_keys=True)
    with open(os.path.join(HERE, "kats.json"), "w") as f:
        json.dump(KATS, f, indent=1, sort_keys=True)
    print("wrote %d vocab configs and %d KATs" % (len(vocab), len(KATS)))


if __name__ == "__main__":
    main()
