"""The reference extension's genetic-operator and tracker exports: mutate_population,
crossover_splicing, constant_perturbation, generate_random_rpn, update_best, check_improvement,
batch_update_best.  CPU: the oracle's properties (valid random programs, same-arity mutation,
splice lengths, the tracker's tie rule).  GPU: identical outputs to the reference extension's
kernels on the same inputs, and to the oracle."""
import numpy as np
import pytest
import torch

import refext
import ws_testlib as tl

O = tl.oracle
gpu = pytest.mark.gpu
needs_ref = pytest.mark.skipif(refext.path("fastmath") is None,
                               reason="reference extension not built (oracle/build_ref.sh)")
DEV = torch.device("cuda:0") if torch.cuda.is_available() else None


def _grammar(V=3):
    return tl.GPUGrammar(num_variables=V, operators=tl.C1_OPERATORS)


def _classes(g):
    ar = np.array(g.arities() + [0], dtype=np.int32)[:g.vocab_size]
    ids = np.arange(g.vocab_size)
    a0 = ids[(ar == 0) & (ids != 0)].astype(np.uint8)
    a1 = ids[ar == 1].astype(np.uint8)
    a2 = ids[ar == 2].astype(np.uint8)
    return ar.astype(np.int32), a0, a1, a2


def _valid(g, pop):
    ar = np.array(g.arities() + [0], dtype=np.int32)
    return O.validate(pop, ar, 0, "kernel")


# ---- CPU (oracle) ------------------------------------------------------------------------
def test_oracle_random_programs_are_valid_and_seeded():
    g = _grammar()
    ar, a0, a1, a2 = _classes(g)
    for L in (1, 2, 7, 30, 64):
        p = O.genrand(3000, L, a0, a1, a2, 12345, 0.4, 0.2, 0.4)
        assert _valid(g, p).all(), L
        assert np.array_equal(p, O.genrand(3000, L, a0, a1, a2, 12345, 0.4, 0.2, 0.4))
    q = O.genrand(3000, 30, a0, a1, a2, 999, 0.4, 0.2, 0.4)
    assert (q != O.genrand(3000, 30, a0, a1, a2, 12345, 0.4, 0.2, 0.4)).any(axis=1).mean() > 0.9
    # no unary operators: still valid (binary/terminal only)
    assert _valid(g, O.genrand(500, 31, a0, a1[:0], a2, 7, 0.5, 0.0, 0.5)).all()


def test_oracle_mutation_keeps_arity():
    g = _grammar()
    ar, a0, a1, a2 = _classes(g)
    rng = np.random.default_rng(1)
    pop = tl.synthetic.random_programs(g, 500, 3, 40, 40, rng, max_consts=4)
    rf = rng.random(pop.shape, dtype=np.float32)
    ri = rng.integers(-2**62, 2**62, size=pop.shape)
    out = O.mutate(pop, rf, ri, ar, a0, a1, a2, 0.3)
    assert _valid(g, out).all()
    changed = out != pop
    assert 0.1 < changed[pop != 0].mean() < 0.3
    assert np.array_equal(ar[out], ar[pop])


def test_oracle_batch_best_tie_rule():
    B, L, K = 600, 8, 3
    rng = np.random.default_rng(2)
    pop = rng.integers(1, 20, size=(B, L)).astype(np.uint8)
    consts = rng.standard_normal((B, K)).astype(np.float32)
    fit = np.full(B, 5.0, np.float32)
    fit[[1, 256, 300]] = 1.0   # thread 0 sees 256 before thread 1 sees 1 in the tree
    rpn, c, r, i = O.batch_best(pop, consts, fit, 1e30)
    assert i == 256 and r == 1.0 and np.array_equal(rpn, pop[256])
    _, _, r2, i2 = O.batch_best(pop, consts, fit, 1.0)  # no improvement
    assert i2 == -1 and r2 == 1.0


# ---- GPU ------------------------------------------------------------------------------------
def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


@gpu
@needs_ref
def test_mutate_population_identical_to_reference():
    from warpsymbolic_b200 import rpn_cuda_native as ours
    ref = refext.load("fastmath")
    g = _grammar(4)
    ar, a0, a1, a2 = _classes(g)
    rng = np.random.default_rng(3)
    pop = tl.synthetic.random_programs(g, 4000, 1, 48, 48, rng, max_consts=4)
    pop[::7, 3] = 250   # tokens outside the table mutate as arity 0
    rf = rng.random(pop.shape, dtype=np.float32)
    ri = rng.integers(-2**63, 2**63 - 1, size=pop.shape, dtype=np.int64)
    outs = []
    for mod in (ref, ours):
        p = T(pop)
        mod.mutate_population(p, T(rf), T(ri), T(ar), T(a0), T(a1), T(a2), 0.25, 0)
        outs.append(p.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
    assert np.array_equal(outs[1], O.mutate(pop, rf, ri, ar, a0, a1, a2, 0.25))
    assert (outs[1] != pop).mean() > 0.05


@gpu
@needs_ref
def test_crossover_splicing_identical_to_reference():
    from warpsymbolic_b200 import rpn_cuda_native as ours
    ref = refext.load("fastmath")
    g = _grammar()
    rng = np.random.default_rng(4)
    N, L = 3000, 40
    p1 = tl.synthetic.random_programs(g, N, 3, L, L, rng, max_consts=4)
    p2 = tl.synthetic.random_programs(g, N, 3, L, L, rng, max_consts=4)
    s1 = rng.integers(-3, L + 3, size=N)
    e1 = s1 + rng.integers(-2, 12, size=N)
    s2 = rng.integers(-3, L + 3, size=N)
    e2 = s2 + rng.integers(-2, 12, size=N)
    mask = rng.random(N) < 0.7
    for m in (None, mask):
        outs = []
        for mod in (ref, ours):
            c1 = torch.empty_like(T(p1))
            c2 = torch.empty_like(T(p2))
            args = [T(p1), T(p2), T(s1), T(e1), T(s2), T(e2), c1, c2, 0]
            if m is not None:
                args.append(T(m))
            mod.crossover_splicing(*args)
            outs.append((c1.cpu().numpy(), c2.cpu().numpy()))
        assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
        w1, w2 = O.splice(p1, p2, s1, e1, s2, e2, m)
        assert np.array_equal(outs[1][0], w1) and np.array_equal(outs[1][1], w2)


@gpu
@needs_ref
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_constant_perturbation_identical_to_reference(dtype):
    from warpsymbolic_b200 import rpn_cuda_native as ours
    ref = refext.load("fastmath")
    rng = np.random.default_rng(5)
    c0 = rng.uniform(-30, 30, size=(5000, 7))
    outs = []
    for mod in (ref, ours):
        c = torch.tensor(c0, dtype=dtype, device=DEV)
        mod.constant_perturbation(c, 0.4, 0.2, -25.0, 25.0, 123456789)
        outs.append(c.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
    base = torch.tensor(c0, dtype=dtype).numpy()
    changed = (outs[1] != base).any(axis=1).mean()
    assert 0.3 < changed < 0.5


@gpu
@needs_ref
@pytest.mark.parametrize("L,weights", [(30, (0.4, 0.2, 0.4)), (64, (0.3, 0.1, 0.6)),
                                       (7, (1.0, 0.0, 1.0)), (1, (0.5, 0.5, 0.5))])
def test_generate_random_rpn_identical_to_reference(L, weights):
    from warpsymbolic_b200 import rpn_cuda_native as ours
    ref = refext.load("fastmath")
    g = _grammar(5)
    _, a0, a1, a2 = _classes(g)
    outs = []
    for mod in (ref, ours):
        p = torch.zeros((20000, L), dtype=torch.uint8, device=DEV)
        mod.generate_random_rpn(p, T(a0), T(a1), T(a2), 2024 + L, *weights)
        outs.append(p.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
    assert _valid(g, outs[1]).all()
    cpu = O.genrand(20000, L, a0, a1, a2, 2024 + L, *weights)
    assert (cpu == outs[1]).all(axis=1).mean() > 0.99   # IEEE vs approximate division


@gpu
@needs_ref
@pytest.mark.parametrize("B", [200, 5000])
def test_best_trackers(B):
    from warpsymbolic_b200 import rpn_cuda_native as ours
    ref = refext.load("fastmath")
    rng = np.random.default_rng(6)
    L, K = 16, 5
    pop8 = rng.integers(0, 30, size=(B, L)).astype(np.uint8)
    consts = rng.standard_normal((B, K)).astype(np.float32)
    fit = rng.uniform(1, 9, size=B).astype(np.float32)
    fit[rng.integers(0, B, size=4)] = 0.5   # ties at the minimum
    fit[rng.integers(0, B, size=4)] = np.nan

    def batch(mod):
        rpn = torch.zeros(L, dtype=torch.uint8, device=DEV)
        bc = torch.zeros(K, dtype=torch.float32, device=DEV)
        br = torch.full((1,), 1e30, dtype=torch.float32, device=DEV)
        bi = torch.full((1,), -1, dtype=torch.int32, device=DEV)
        mod.batch_update_best(T(pop8), T(consts), T(fit), rpn, bc, br, bi)
        return rpn.cpu().numpy(), bc.cpu().numpy(), float(br.item()), int(bi.item())

    a, b = batch(ref), batch(ours)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    w = O.batch_best(pop8, consts, fit, 1e30)
    assert b[3] == w[3] and b[2] == w[2]

    def upd(mod):
        t = [torch.zeros(L, dtype=torch.int64, device=DEV), torch.zeros(K, dtype=torch.float32, device=DEV),
             torch.full((1,), 1e30, dtype=torch.float32, device=DEV)] + \
            [torch.zeros(1, dtype=torch.int32, device=DEV) for _ in range(4)]
        mod.update_best(T(pop8.astype(np.int64)), T(consts), T(fit), *t, 7)
        imp = torch.zeros(1, dtype=torch.int32, device=DEV)
        mod.check_improvement(T(fit), torch.full((1,), 0.75, dtype=torch.float32, device=DEV), imp)
        return [x.cpu().numpy() for x in t] + [imp.cpu().numpy()]

    ours_u = upd(ours)
    assert float(ours_u[2][0]) == 0.5 and int(ours_u[4][0]) == 7 and int(ours_u[6][0]) == 1
    assert int(ours_u[7][0]) == 1
    if B <= 256:  # one block in the reference too: the same bits
        ref_u = upd(ref)
        assert all(np.array_equal(x, y) for x, y in zip(ref_u, ours_u))
