"""Generates tests/golden/ref_decode.json: outputs of the REFERENCE's decode_rpn
(decoder.cpp:32-152, a host function of its extension), called on the CPU through the extension
built from the reference's sources by oracle/build_ref.sh.

Cases: the grammar's own vocabularies (all operators, three variables) with valid programs,
malformed ones (underflow, leftovers, tokens outside the vocabulary, PAD gaps), constants of
every shape format_const distinguishes (integral, negative, tiny, large, rounding to zero, NaN,
inf, more C tokens than constants), several precisions, and a vocabulary with the decoder's
aliases ("x", "s", "^", "mod", "!") and an arity-3 token.

Usage: python tests/golden/make_decode_golden.py   (needs oracle/_ref; no GPU)
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import refext  # noqa: E402
import ws_testlib as tl  # noqa: E402


def cases():
    rng = np.random.default_rng(77)
    out = []
    g = tl.GPUGrammar(num_variables=3, operators=tl.ALL_OPERATORS)
    vocab = [g.id_to_token.get(i, "") for i in range(g.vocab_size)]
    arities = [0] * g.vocab_size
    for t, a in enumerate(g.arities()):
        arities[t] = a
    pop, _ = tl.random_population(g, 300, 24, 4, rng, valid_only=False)
    specials = np.array([0.0, -0.0, 3.0, -7.0, 2.5, -0.00001, 1e-12, 123456.789, 1e12 + 0.5,
                         0.49999, 1.23456789, -2.0000000001, np.nan, np.inf, -np.inf],
                        dtype=np.float64)
    for prec in (4, 2, 0, 8):
        for dt in ("float32", "float64"):
            consts = rng.uniform(-10, 10, size=(300, 4))
            consts[::3] = rng.choice(specials, size=(100, 4))
            out.append({"vocab": vocab, "arities": arities, "pad": 0, "precision": prec,
                        "dtype": dt, "population": pop.tolist(),
                        "constants": consts.astype(dt).tolist()})
    # alias vocabulary: ids 1.. with single-letter aliases and an arity-3 token
    vocab2 = ["", "x", "C", "s", "c", "^", "mod", "!", "neg", "T", "tri", "zz", "e", "q", "+"]
    ar2 = [0, 0, 0, 1, 1, 2, 2, 1, 1, 1, 3, 5, 1, 1, 2]
    pop2 = rng.integers(0, 18, size=(400, 12)).astype(np.uint8)
    pop2[:, 0] = rng.integers(1, 3, size=400)
    consts2 = rng.uniform(-3, 3, size=(400, 3))
    out.append({"vocab": vocab2, "arities": ar2, "pad": 0, "precision": 3, "dtype": "float64",
                "population": pop2.tolist(), "constants": consts2.tolist()})
    return out


def main():
    ref = refext.load("fastmath")
    if ref is None:
        raise SystemExit("reference extension not built (oracle/build_ref.sh)")
    recs = []
    for c in cases():
        pop = torch.tensor(c["population"], dtype=torch.uint8)
        cst = torch.tensor(c["constants"], dtype=getattr(torch, c["dtype"]))
        c["expected"] = ref.decode_rpn(pop, cst, c["vocab"], c["arities"], c["pad"],
                                       c["precision"])
        recs.append(c)
    with open(os.path.join(HERE, "ref_decode.json"), "w") as f:
        json.dump(recs, f, allow_nan=True)
    print("wrote", len(recs), "cases")


if __name__ == "__main__":
    main()
