"""decode_rpn (host-side RPN -> infix text) against the reference's own decoder: the committed
fixture golden/ref_decode.json (recorded by golden/make_decode_golden.py with the reference
extension built from source), and live against that extension when it is present."""
import json
import os

import numpy as np
import pytest
import torch

import refext
import ws_testlib as tl

HERE = os.path.dirname(os.path.abspath(__file__))


def _cases():
    with open(os.path.join(HERE, "golden", "ref_decode.json")) as f:
        return json.load(f)


def test_decode_matches_reference_fixture():
    from warpsymbolic_b200 import rpn_cuda_native as ours
    n = 0
    for c in _cases():
        pop = torch.tensor(c["population"], dtype=torch.uint8)
        cst = torch.tensor(c["constants"], dtype=getattr(torch, c["dtype"]))
        got = ours.decode_rpn(pop, cst, c["vocab"], c["arities"], c["pad"], c["precision"])
        assert got == c["expected"], [(i, a, b) for i, (a, b) in
                                      enumerate(zip(got, c["expected"])) if a != b][:3]
        n += len(got)
    assert n >= 2800


def test_decode_known_strings():
    from warpsymbolic_b200 import rpn_cuda_native as ours
    g = tl.GPUGrammar(num_variables=2, operators=tl.ALL_OPERATORS)
    vocab = [g.id_to_token.get(i, "") for i in range(g.vocab_size)]
    ar = g.arities()
    rows = [["x0", "C", "*", "sin"], ["C", "C", "+"], ["x0", "x1"], ["+"], ["x1", "neg"]]
    pop = torch.tensor([g.encode(r, 6) for r in rows], dtype=torch.uint8)
    cst = torch.tensor([[2.5, 0], [3.0, -0.00001], [0, 0], [0, 0], [0, 0]], dtype=torch.float64)
    assert ours.decode_rpn(pop, cst, vocab, ar, 0) == [
        "sin((x0 * 2.5))", "(3 + -0)", "Invalid", "Invalid", "neg(x1)"]


@pytest.mark.skipif(refext.path("fastmath") is None, reason="reference extension not built")
def test_decode_live_against_reference():
    ref = refext.load("fastmath")
    from warpsymbolic_b200 import rpn_cuda_native as ours
    rng = np.random.default_rng(5)
    g = tl.GPUGrammar(num_variables=4, operators=tl.ALL_OPERATORS)
    vocab = [g.id_to_token.get(i, "") for i in range(g.vocab_size)]
    pop, consts = tl.random_population(g, 2000, 40, 6, rng, valid_only=False)
    P = torch.from_numpy(pop)
    for dt in (torch.float32, torch.float64):
        C = torch.from_numpy(consts).to(dt) * 7
        for prec in (0, 4, 6):
            assert ours.decode_rpn(P, C, vocab, g.arities(), 0, prec) == \
                ref.decode_rpn(P, C, vocab, g.arities(), 0, prec)
