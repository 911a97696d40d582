"""The generator tables of population.PopulationOperators against the reference's own
GPUOperators (src/warpsymbolic/gpu/operators.py:17-236), both built on the CPU: token arities,
terminal IDs, the prior-weighted operator ID lists, the category weights and the native seed
sequence.  The reference runs in a subprocess (its package binds the native module at import).
Skipped when the reference package is not installed in baseline/_ref."""
import json
import os
import subprocess
import sys

import pytest
import torch

import ws_testlib as tl

REF_PKG = os.path.join(tl.REPO, "baseline", "_ref")
pytestmark = pytest.mark.skipif(not os.path.isdir(os.path.join(REF_PKG, "warpsymbolic")),
                                reason="reference package not installed in baseline/_ref")

SCRIPT = r'''
import json, sys, torch
sys.path.insert(0, sys.argv[1])
from warpsymbolic.gpu.config import GpuGlobals
GpuGlobals.USE_OP_POW = sys.argv[3] == "1"
GpuGlobals.USE_OP_ABS = sys.argv[3] == "1"
GpuGlobals.USE_OP_GAMMA = sys.argv[3] == "1"
from warpsymbolic.gpu.grammar import GPUGrammar
from warpsymbolic.gpu.operators import GPUOperators
torch.manual_seed(int(sys.argv[4]))
nv = int(sys.argv[2])
ops = GPUOperators(GPUGrammar(nv), torch.device("cpu"), 64, 30, nv, dtype=torch.float32)
g = ops.grammar
print(json.dumps({"vocab": [g.id_to_token[i] for i in sorted(g.id_to_token)],
                  "arity": ops.token_arity.tolist(), "terminals": ops.terminal_ids.tolist(),
                  "a1": ops.arity_1_ids.tolist(), "a2": ops.arity_2_ids.tolist(),
                  "weights": list(ops._sampling_category_weights()),
                  "seeds": [ops._next_native_seed(s) for s in (0, 0xA341316C, 7)]}))
'''


@pytest.mark.parametrize("nv,extra", [(2, "0"), (3, "1"), (1, "0")])
def test_tables_match_reference(nv, extra):
    from warpsymbolic_b200.population import PopulationOperators
    seed = 1234 + nv
    out = subprocess.run([sys.executable, "-c", SCRIPT, REF_PKG, str(nv), extra, str(seed)],
                         capture_output=True, text=True, timeout=300, cwd="/")
    assert out.returncode == 0, out.stderr[-3000:]
    ref = json.loads(out.stdout.strip().splitlines()[-1])
    ops_names = [t for t in ref["vocab"][1:] if t not in tl.GPUGrammar(nv).terminals]
    g = tl.GPUGrammar(num_variables=nv, operators=[o for o in ops_names if o != 'neg'])
    assert [g.id_to_token[i] for i in sorted(g.id_to_token)] == ref["vocab"]
    torch.manual_seed(seed)
    ops = PopulationOperators(g, "cpu", 30, nv)
    assert ops.token_arity.tolist() == ref["arity"]
    assert ops.terminal_ids.tolist() == ref["terminals"]
    assert ops.arity_1_ids.tolist() == ref["a1"]
    assert ops.arity_2_ids.tolist() == ref["a2"]
    assert list(ops.category_weights()) == ref["weights"]
    assert [ops.next_native_seed(s) for s in (0, 0xA341316C, 7)] == ref["seeds"]
