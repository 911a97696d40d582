"""simplify_batch: the rule-based rewriter.  CPU: the oracle (a literal restatement of the
reference kernel) on hand cases and against the reference kernel's recorded outputs
(golden/ref_simplify.npz); GPU: identical programs to the reference extension's kernel on the
same inputs, agreement with the oracle, and the GPUSymbolicSimplifier wrapper's rules."""
import os

import numpy as np
import pytest
import torch

import refext
import ws_testlib as tl

O = tl.oracle
HERE = os.path.dirname(os.path.abspath(__file__))
gpu = pytest.mark.gpu
needs_ref = pytest.mark.skipif(refext.path("fastmath") is None,
                               reason="reference extension not built (oracle/build_ref.sh)")
DEV = torch.device("cuda:0") if torch.cuda.is_available() else None


def _tables(g):
    from warpsymbolic_b200.simplifier import GPUSymbolicSimplifier
    s = GPUSymbolicSimplifier(g, "cpu")
    return (s.arity_table.numpy(), s.val_table.numpy(), s.literal_ids.numpy(),
            s.literal_vals.numpy(), np.array(s.op_ids, dtype=np.int32))


def literal_rich(g, B, L, seed, frac=0.4):
    """Valid programs (no C) in which `frac` of the terminals are literals 0, 1, 2, ... so that
    identity, zero, folding and normalisation rules fire often."""
    rng = np.random.default_rng(seed)
    pop = tl.synthetic.random_programs(g, B, 1, L, L, rng, const_prob=0.0,
                                       use_literals=True).astype(np.int64)
    ar = np.array(g.arities(), dtype=np.int32)
    lits = np.array([g.token_to_id[t] for t in ('0', '1', '2', '3', 'pi')], dtype=np.int64)
    term = (pop != 0) & (ar[pop] == 0)
    pick = term & (rng.random(pop.shape) < frac)
    pop[pick] = lits[rng.integers(0, len(lits), size=int(pick.sum()))]
    return pop


def _simplify_oracle(g, pop, passes=3):
    ar, vt, li, lv, ids = _tables(g)
    return O.simplify(pop, ar, vt, li, lv, passes, ids)


def test_oracle_hand_cases():
    g = tl.GPUGrammar(num_variables=2, operators=tl.ALL_OPERATORS)
    cases = [
        (["x0", "0", "+"], ["x0"]),
        (["x0", "1", "*"], ["x0"]),
        (["1", "x0", "*"], ["x0"]),
        (["x0", "0", "*"], ["0"]),
        (["0", "x0", "-"], ["x0", "neg"]),
        (["x0", "neg", "neg"], ["x0"]),
        (["x0", "2", "pow", "sqrt"], ["x0", "abs"]),
        (["0", "sin"], ["0"]),
        (["0", "cos"], ["1"]),
        (["x0", "x0", "neg", "+"], ["0"]),
        (["2", "3", "+"], ["5"]),
        (["x1", "x0", "+"], ["x0", "x1", "+"]),          # operands ordered by token ID
        (["x0", "3", "*"], ["3", "x0", "*"]),            # literal before variable
        # x + (y + x) -> 2 x * y + ; a later pass orders the + operands (single token first)
        (["x0", "x1", "x0", "+", "+"], ["x1", "2", "x0", "*", "+"]),
        (["2", "x0", "*", "3", "x0", "*", "+"], ["5", "x0", "*"]),  # factor, then fold 2 + 3
        (["x0", "x0", "-"], ["x0", "x0", "-"]),          # domain-sensitive rules stay off
    ]
    L = 10
    pop = np.array([g.encode(a, L) for a, _ in cases], dtype=np.int64)
    out = _simplify_oracle(g, pop, passes=5)
    for (src, want), row in zip(cases, out):
        assert row.tolist() == g.encode(want, L), (src, [g.id_to_token[int(t)] for t in row if t])


def test_oracle_matches_reference_kernel_fixture():
    p = os.path.join(HERE, "golden", "ref_simplify.npz")
    if not os.path.exists(p):
        pytest.skip("fixture not recorded")
    z = np.load(p)
    for passes in (1, 3):
        got = O.simplify(z["population"], z["arities"], z["val_table"], z["literal_ids"],
                         z["literal_vals"], passes, z["ids"])
        want = z["out_p%d" % passes]
        same = (got == want).all(axis=1)
        # host libm vs the reference's fast-math folding: only rows whose folded value sits at
        # the 1e-5 acceptance edge may differ
        assert same.mean() > 0.999, np.nonzero(~same)[0][:5]


@gpu
@needs_ref
@pytest.mark.parametrize("L,passes", [(30, 3), (64, 5), (256, 3), (300, 2)])
def test_simplify_identical_to_reference(L, passes):
    ref = refext.load("fastmath")
    from warpsymbolic_b200 import rpn_cuda_native as ours
    g = tl.GPUGrammar(num_variables=3, operators=tl.ALL_OPERATORS)
    B = 4000
    pop = literal_rich(g, B, min(L, 256), 100 + L)
    if L > 256:  # positions beyond 256 are left alone
        pad = np.random.default_rng(1).integers(1, 20, size=(B, L - 256))
        pop = np.concatenate([pop, pad], axis=1)
    ar, vt, li, lv, ids = _tables(g)
    args = [torch.from_numpy(a).to(DEV) for a in (ar, vt, li, lv)]
    outs = []
    for mod in (ref, ours):
        t = torch.from_numpy(pop.copy()).to(DEV)
        mod.simplify_batch(t, *args, passes, *[int(v) for v in ids])
        outs.append(t.cpu().numpy())
    torch.cuda.synchronize()
    diff = np.nonzero((outs[0] != outs[1]).any(axis=1))[0]
    assert diff.size == 0, diff[:5]
    assert (outs[1] != pop).any(axis=1).mean() > 0.3   # the rules really fired
    want = _simplify_oracle(g, pop, passes)
    assert (want == outs[1]).all(axis=1).mean() > 0.999


@gpu
def test_wrapper_rules():
    """Rows holding C stay unchanged; the others are simplified; results stay stack-valid."""
    from warpsymbolic_b200.simplifier import GPUSymbolicSimplifier
    from warpsymbolic_b200.structure import validate_population
    g = tl.GPUGrammar(num_variables=2, operators=tl.C1_OPERATORS)
    pop = literal_rich(g, 2000, 40, 7).astype(np.uint8)
    c_id = g.token_to_id["C"]
    rows_c = np.arange(0, 2000, 5)
    pop[rows_c, 0] = np.where(np.array(g.arities())[pop[rows_c, 0]] == 0, c_id, pop[rows_c, 0])
    has_c = (pop == c_id).any(axis=1)
    s = GPUSymbolicSimplifier(g, DEV)
    P = torch.from_numpy(pop).to(DEV)
    consts = torch.randn(2000, 4, device=DEV)
    out, c_out, _ = s.simplify_batch(P, consts, max_passes=3)
    o = out.cpu().numpy()
    assert np.array_equal(o[has_c], pop[has_c])
    assert (o[~has_c] != pop[~has_c]).any(axis=1).mean() > 0.3
    assert torch.equal(c_out, consts)
    ar = torch.tensor(g.arities(), dtype=torch.int32, device=DEV)
    v_in = validate_population(P, ar, 0, "stack")
    v_out = validate_population(out, ar, 0, "stack")
    assert bool((v_out | ~v_in).all())


@gpu
def test_wide_tokens_take_the_same_rules():
    """A row holding a token outside the 16-bit range is rewritten from an int64 copy: the same
    rows with an out-of-vocabulary token of 200 (16-bit path) or 40000 (int64 path) at the same
    positions simplify identically, and both agree with the oracle."""
    from warpsymbolic_b200 import rpn_cuda_native as ours
    g = tl.GPUGrammar(num_variables=3, operators=tl.ALL_OPERATORS)
    B, L = 3000, 48
    pop = literal_rich(g, B, L, 5)
    rng = np.random.default_rng(6)
    rows = rng.random(B) < 0.5
    cols = rng.integers(0, L, size=B)
    narrow, wide = pop.copy(), pop.copy()
    narrow[rows, cols[rows]] = 200
    wide[rows, cols[rows]] = 40000
    wide[3, 0] = -(1 << 40)   # and one far outside
    narrow[3, 0] = -7
    ar, vt, li, lv, ids = _tables(g)
    args = [torch.from_numpy(a).to(DEV) for a in (ar, vt, li, lv)]
    outs = []
    for p in (narrow, wide):
        t = torch.from_numpy(p.copy()).to(DEV)
        ours.simplify_batch(t, *args, 3, *[int(v) for v in ids])
        outs.append(t.cpu().numpy())
    back = outs[1].copy()
    back[back == 40000] = 200
    back[back == -(1 << 40)] = -7
    assert np.array_equal(outs[0], back)
    assert (outs[1] != wide).any(axis=1).mean() > 0.3
    want = _simplify_oracle(g, wide, 3)
    assert (want == outs[1]).all(axis=1).mean() > 0.999
