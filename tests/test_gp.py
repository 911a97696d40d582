"""Device GP generations (ws_gp_*): CPU oracle properties (valid children from valid parents,
elitism, determinism, length bound, inherited constants) and, on the GPU, child-by-child
agreement with the oracle, independence from the other problems of a launch, and graph replay
with the device-side generation counter."""
import numpy as np
import pytest
import torch

import ws_testlib as tl

O = tl.oracle
gpu = pytest.mark.gpu
DEV = torch.device("cuda:0") if torch.cuda.is_available() else None
OPTS = dict(tournament_size=3, elitism=1, crossover_rate=0.7, mutation_rate=0.08,
            const_mutation_rate=0.2, const_sigma=0.1, parsimony_eps=1e-9)


def _case(seed, B=400, L=40, V=3, K=6, dtype=np.float32):
    rng = np.random.default_rng(seed)
    g = tl.GPUGrammar(num_variables=V, operators=tl.C1_OPERATORS)
    pop = tl.synthetic.random_programs(g, B, 3, L, L, rng, max_consts=K)
    consts = rng.uniform(-2, 2, size=(B, K)).astype(dtype)
    fit = rng.uniform(0, 10, size=B).astype(dtype)
    fit[rng.integers(0, B, size=5)] = np.nan
    return g, pop, consts, fit


def _valid(g, pop):
    ar = np.array(g.arities() + [0], dtype=np.int32)
    return O.validate(pop, ar, 0, "kernel")


def test_oracle_children_are_valid_and_elite_first():
    g, pop, consts, fit = _case(1)
    assert _valid(g, pop).all()
    cp, cc = O.gp_step(g, pop, consts, fit, seed=7, generation=0, **OPTS)
    assert _valid(g, cp).all()
    best = int(np.nanargmin(fit))
    assert np.array_equal(cp[0], pop[best]) and np.array_equal(cc[0], consts[best])
    # deterministic per (seed, generation); a new generation draws differently
    cp2, cc2 = O.gp_step(g, pop, consts, fit, seed=7, generation=0, **OPTS)
    assert np.array_equal(cp, cp2) and np.array_equal(cc, cc2)
    cp3, _ = O.gp_step(g, pop, consts, fit, seed=7, generation=1, **OPTS)
    assert (cp3 != cp).any(axis=1).mean() > 0.5


def test_oracle_copies_without_variation():
    """No crossover, no mutation, tournament of one: every child is one program of the
    population, unchanged, with that program's constants."""
    g, pop, consts, fit = _case(2)
    o = dict(OPTS, crossover_rate=0.0, mutation_rate=0.0, const_mutation_rate=0.0,
             tournament_size=1, elitism=0)
    cp, cc = O.gp_step(g, pop, consts, fit, seed=3, generation=5, **o)
    rows = {(pop[i].tobytes(), consts[i].tobytes()) for i in range(len(pop))}
    assert all((cp[i].tobytes(), cc[i].tobytes()) in rows for i in range(len(cp)))
    assert len({cp[i].tobytes() for i in range(len(cp))}) > 0.5 * len(cp)


def test_oracle_mutation_rate_and_selection_pressure():
    g, pop, consts, fit = _case(3, B=3000)
    fit = np.arange(len(pop), dtype=np.float32)[np.random.default_rng(0).permutation(len(pop))]
    o = dict(OPTS, crossover_rate=0.0, mutation_rate=0.0, const_mutation_rate=0.0, elitism=0)
    cp, _ = O.gp_step(g, pop, consts, fit, seed=11, generation=0, **o)
    # selected parents: the fitness of the chosen rows is well below the population mean
    rows = {pop[i].tobytes(): fit[i] for i in range(len(pop))}
    sel = np.array([rows[r.tobytes()] for r in cp])
    # tournament of 3 over uniform ranks: the expected winner sits at a quarter of the range
    assert 0.4 * fit.mean() < sel.mean() < 0.6 * fit.mean()
    # mutation: changed operator / variable tokens close to the rate x (1 - 1/choices)
    o2 = dict(o, mutation_rate=0.1, tournament_size=1)
    a, _ = O.gp_step(g, pop, consts, fit, seed=11, generation=0, **dict(o2, mutation_rate=0.0))
    b, _ = O.gp_step(g, pop, consts, fit, seed=11, generation=0, **o2)
    changed = (a != b).sum() / max(1, (a != 0).sum())
    assert 0.02 < changed < 0.1


def test_oracle_length_bound_and_constants_inherited():
    g, pop, consts, fit = _case(4, L=24)
    cp, cc = O.gp_step(g, pop, consts, fit, seed=5, generation=2, **dict(OPTS, const_mutation_rate=0.0))
    assert cp.shape == pop.shape and _valid(g, cp).all()
    pool = set(np.round(consts.ravel().astype(np.float64), 7))
    assert all(np.round(float(v), 7) in pool for v in cc.ravel())


def _gpu_problems(seeds, **kw):
    from warpsymbolic_b200.batch import BatchProblem
    out, host = [], []
    for s in seeds:
        g, pop, consts, fit = _case(s, **kw)
        X = np.zeros((len(g.active_variables), 8), dtype=consts.dtype)
        out.append(BatchProblem(torch.from_numpy(pop).to(DEV), torch.from_numpy(X).to(DEV),
                                torch.zeros(8, dtype=torch.float32 if consts.dtype == np.float32
                                            else torch.float64, device=DEV),
                                torch.from_numpy(consts).to(DEV), g))
        host.append((g, pop, consts, fit))
    return out, host


@gpu
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_gpu_step_matches_oracle(dtype):
    from warpsymbolic_b200.gp import GPStep
    probs, host = _gpu_problems([21, 22, 23], dtype=dtype)
    fits = [torch.from_numpy(h[3]).to(DEV) for h in host]
    seeds = [101, 202, 303]
    gp = GPStep(probs, fits, seeds, **{k: v for k, v in OPTS.items()})
    for gen in range(3):
        want = [O.gp_step(h[0], p.population.cpu().numpy(), p.constants.cpu().numpy(), h[3],
                          seed=s, generation=gen, **OPTS) for p, h, s in zip(probs, host, seeds)]
        gp.step()
        torch.cuda.synchronize()
        for p, (wp, wc) in zip(probs, want):
            assert np.array_equal(p.population.cpu().numpy(), wp)
            np.testing.assert_allclose(p.constants.cpu().numpy(), wc, rtol=1e-6 if dtype == np.float32 else 1e-12)
    gp.close()


@gpu
def test_gpu_step_independent_of_other_problems():
    from warpsymbolic_b200.gp import GPStep
    probs, host = _gpu_problems([31, 32, 33, 34])
    alone, h1 = _gpu_problems([33])
    fits = [torch.from_numpy(h[3]).to(DEV) for h in host]
    GPStep(probs, fits, [1, 2, 3, 4], **OPTS).step()
    GPStep(alone, [fits[2]], [3], **OPTS).step()
    torch.cuda.synchronize()
    assert torch.equal(probs[2].population, alone[0].population)
    assert torch.equal(probs[2].constants, alone[0].constants)


@gpu
def test_gpu_evaluate_and_step_graph_replay():
    """evaluate + breed captured once; each replay is one generation (the counter advances on
    the device), equal to the same generations run eagerly."""
    from warpsymbolic_b200.batch import BatchProblem, BatchedFitness
    from warpsymbolic_b200.gp import GPStep
    rng = np.random.default_rng(9)

    def build():
        probs = []
        for i in range(3):
            g = tl.GPUGrammar(num_variables=2, operators=tl.C1_OPERATORS)
            r = np.random.default_rng(40 + i)
            pop = tl.synthetic.random_programs(g, 256, 3, 30, 30, r, max_consts=4)
            X = r.uniform(-2, 2, size=(2, 300)).astype(np.float32)
            y = (X[0] ** 2 + np.sin(X[1])).astype(np.float32)
            c = r.uniform(-2, 2, size=(256, 4)).astype(np.float32)
            probs.append(BatchProblem(torch.from_numpy(pop).to(DEV), torch.from_numpy(X).to(DEV),
                                      torch.from_numpy(y).to(DEV), torch.from_numpy(c).to(DEV), g))
        bf = BatchedFitness(probs, loss="mse", policy="classic")
        gp = GPStep(probs, bf.outputs, [5, 6, 7], **OPTS)
        return probs, bf, gp

    pa, bfa, gpa = build()
    for _ in range(3):
        bfa.evaluate()
        gpa.step()
    bfa.evaluate()
    torch.cuda.synchronize()
    pb, bfb, gpb = build()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    graph = torch.cuda.CUDAGraph()
    saved = [(p.population.clone(), p.constants.clone()) for p in pb]
    with torch.cuda.stream(s):  # warm-up outside capture, then restore and rewind the counter
        bfb.evaluate(stream=s)
        gpb.step(stream=s)
        for p, (sp, sc) in zip(pb, saved):
            p.population.copy_(sp)
            p.constants.copy_(sc)
        gpb.set_generation(0, stream=s)
    torch.cuda.current_stream().wait_stream(s)
    with torch.cuda.graph(graph):
        bfb.evaluate()
        gpb.step()
    for _ in range(3):
        graph.replay()
    bfb.evaluate()
    torch.cuda.synchronize()
    for a, b in zip(pa, pb):
        assert torch.equal(a.population, b.population)
        assert torch.equal(a.constants, b.constants)
    for a, b in zip(bfa.outputs, bfb.outputs):
        assert torch.equal(a, b)
    assert min(float(o.min()) for o in bfb.outputs) < 1e15
    del graph
