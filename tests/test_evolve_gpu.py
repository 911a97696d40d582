"""evolve_generation drop-in against the reference extension's own evolve_generation: with the
same inputs and the same torch seed, the new population, its constants and the PSO fitness are
identical (bytes and float bits), across the selection variants (tournament, lexicase cases with
MAD epsilons, islands), with and without a mutation bank, with and without PSO."""
import math

import numpy as np
import pytest
import torch

import refext
import ws_testlib as tl
from test_gpops import _classes

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(refext.path("fastmath") is None,
                               reason="reference extension not built (oracle/build_ref.sh)")
DEV = torch.device("cuda:0") if torch.cuda.is_available() else None


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def _case(seed, B, L, K, D, V=3, bank=0):
    rng = np.random.default_rng(seed)
    g = tl.GPUGrammar(num_variables=V, operators=tl.C1_OPERATORS)
    pop = tl.synthetic.random_programs(g, B, 2, L, L, rng, const_prob=0.4, max_consts=K)
    consts = rng.uniform(-2, 2, size=(B, K)).astype(np.float32)
    X = rng.uniform(-2, 2, size=(V, D)).astype(np.float32)
    y = (np.sin(X[0]) + X[1] * X[2]).astype(np.float32)
    fit = rng.uniform(0.1, 5.0, size=B).astype(np.float32)
    fit[rng.integers(0, B, size=B // 20)] = 2.5  # ties
    lengths = (pop != 0).sum(1).astype(np.float32)
    bank_rows = tl.synthetic.random_programs(g, bank, 2, L, L, rng, max_consts=K) if bank else None
    return g, pop, consts, X, y, fit, lengths, bank_rows, rng


def _run(mod, g, pop, consts, X, y, fit, lengths, bank, abs_err, mad, mrate, crate, tsize,
         steps, parts, n_islands, seed, gen):
    ar, a0, a1, a2 = _classes(g)
    e64 = torch.empty(0, dtype=torch.int64, device=DEV)
    ef = torch.empty(0, dtype=torch.float32, device=DEV)
    ids = g.scalar_ids()
    torch.manual_seed(seed)
    out = mod.evolve_generation(
        T(pop), T(consts), T(fit), T(abs_err) if abs_err is not None else ef, T(X), T(y),
        T(lengths), T(ar), T(a0), T(a1), T(a2),
        T(bank) if bank is not None else torch.empty(0, dtype=torch.uint8, device=DEV),
        T(mad) if mad is not None else ef, mrate, crate, tsize, steps, parts, 0.5, 1.5, 1.5,
        *ids, 3.14159265359, 2.718281828, n_islands, e64, e64, e64, e64, 12345 + seed, gen)
    return [o.cpu().numpy() for o in out]


CASES = [
    # (B, L, K, D, bank, errors, islands, pso_steps, particles, mutation, crossover, tsize)
    (1000, 30, 6, 64, 0, False, 1, 0, 0, 0.15, 0.7, 3),
    (1024, 40, 8, 96, 64, True, 4, 3, 6, 0.2, 0.5, 4),
    (777, 24, 4, 48, 32, False, 3, 2, 4, 0.3, 0.9, 2),
]


@needs_ref
@pytest.mark.parametrize("case", CASES)
def test_evolve_generation_identical_to_reference(case):
    from warpsymbolic_b200 import rpn_cuda_native as ours
    ref = refext.load("fastmath")
    B, L, K, D, bank_n, with_err, islands, steps, parts, mrate, crate, tsize = case
    g, pop, consts, X, y, fit, lengths, bank, rng = _case(B + L, B, L, K, D, bank=bank_n)
    abs_err = mad = None
    if with_err:
        abs_err = np.abs(rng.standard_normal((B, D))).astype(np.float32)
        mad = (0.05 * np.abs(rng.standard_normal(D))).astype(np.float32)
    for gen in (0, 7):
        r = _run(ref, g, pop, consts, X, y, fit, lengths, bank, abs_err, mad, mrate, crate, tsize,
                 steps, parts, islands, 5, gen)
        o = _run(ours, g, pop, consts, X, y, fit, lengths, bank, abs_err, mad, mrate, crate,
                 tsize, steps, parts, islands, 5, gen)
        assert np.array_equal(r[0], o[0]), (gen, int((r[0] != o[0]).sum()))
        assert np.array_equal(r[1].view(np.uint32), o[1].view(np.uint32)), gen
        assert np.array_equal(r[2].view(np.uint32), o[2].view(np.uint32)), gen
        assert (o[0] != pop).any()  # something changed
        if steps:
            assert o[2].shape == (B,) and np.isfinite(o[2]).mean() > 0.5
        else:
            assert o[2].size == 0
