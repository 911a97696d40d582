"""Speed of every exported kernel against the reference extension's own kernel on identical
inputs (B200, CUDA events, median of 5 after 2 warm-up calls).  Records the table in
the output folder's reference_speed_all.json (when that folder exists) and asserts that no
export is slower than the reference's by more than timing noise."""
import math
import statistics

import numpy as np
import pytest
import torch

import refext
import ws_testlib as tl
from test_gpops import _classes
from test_simplify import _tables, literal_rich

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(refext.path("fastmath") is None,
                               reason="reference extension not built (oracle/build_ref.sh)")
DEV = torch.device("cuda:0") if torch.cuda.is_available() else None


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def _time(fn, reps=5):
    for _ in range(2):
        fn()
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        ms.append(a.elapsed_time(b))
    return statistics.median(ms)


def _cases():
    """name -> callable(mod) -> work closure, for every export with a reference kernel."""
    rng = np.random.default_rng(0)
    g = tl.GPUGrammar(num_variables=3, operators=tl.C1_OPERATORS)
    ids = g.scalar_ids()
    ar, a0, a1, a2 = _classes(g)
    cases = {}

    B1, L1 = 1 << 20, 64
    pop1 = tl.synthetic.random_programs(g, B1, 3, L1, L1, rng, max_consts=8)
    P1, A = T(pop1), T(ar)
    valid = torch.empty(B1, dtype=torch.bool, device=DEV)
    cases["validate_rpn_batch (1M x 64)"] = lambda m: (lambda: m.validate_rpn_batch(P1, A, valid, 0))
    starts = torch.empty((B1, L1), dtype=torch.int64, device=DEV)
    lens = torch.empty(B1, dtype=torch.int64, device=DEV)
    cases["find_subtree_ranges (1M x 64)"] = lambda m: (
        lambda: m.find_subtree_ranges(P1, A, starts, 0, lens))
    P64 = T(pop1[:1 << 18].astype(np.int64))
    pre = torch.empty((1 << 18, L1), dtype=torch.int64, device=DEV)
    cases["precompute_subtree_starts (256K x 64)"] = lambda m: (
        lambda: m.precompute_subtree_starts(P64, A, pre))
    fit = T(rng.uniform(0, 5, B1).astype(np.float32))
    cand = T(rng.integers(0, B1, size=(B1, 4)).astype(np.int64))
    e0 = torch.empty(0, dtype=torch.float32, device=DEV)
    i0 = torch.empty(0, dtype=torch.int32, device=DEV)
    lens_f = T((pop1 != 0).sum(1).astype(np.float32))
    win = torch.empty(B1, dtype=torch.int64, device=DEV)
    cases["tournament_selection (1M, size 4)"] = lambda m: (
        lambda: m.tournament_selection(fit, e0, cand, i0, win, lens_f, e0))
    rf = T(rng.random(pop1.shape, dtype=np.float32))
    ri = T(rng.integers(-2**63, 2**63 - 1, size=pop1.shape, dtype=np.int64))
    Pm = P1.clone()
    cases["mutate_population (1M x 64)"] = lambda m: (
        lambda: m.mutate_population(Pm, rf, ri, A, T(a0), T(a1), T(a2), 0.05, 0))
    N = 1 << 19
    p1, p2 = P1[:N], P1[N:2 * N]
    s1 = T(rng.integers(0, 8, N).astype(np.int64))
    e1 = s1 + 2
    s2 = T(rng.integers(0, 8, N).astype(np.int64))
    e2 = s2 + 3
    c1, c2 = torch.empty_like(p1), torch.empty_like(p2)
    cases["crossover_splicing (512K pairs x 64)"] = lambda m: (
        lambda: m.crossover_splicing(p1, p2, s1, e1, s2, e2, c1, c2, 0))
    cst = T(rng.uniform(-2, 2, (B1, 8)).astype(np.float32))
    cases["constant_perturbation (1M x 8)"] = lambda m: (
        lambda: m.constant_perturbation(cst, 0.3, 0.1, -25.0, 25.0, 7))
    Pg = torch.empty((B1, L1), dtype=torch.uint8, device=DEV)
    cases["generate_random_rpn (1M x 64)"] = lambda m: (
        lambda: m.generate_random_rpn(Pg, T(a0), T(a1), T(a2), 11, 0.45, 0.15, 0.40))
    rpn = torch.zeros(L1, dtype=torch.uint8, device=DEV)
    bc = torch.zeros(8, dtype=torch.float32, device=DEV)
    br = torch.full((1,), 1e30, dtype=torch.float32, device=DEV)
    bi = torch.full((1,), -1, dtype=torch.int32, device=DEV)
    cases["batch_update_best (1M)"] = lambda m: (
        lambda: m.batch_update_best(P1, cst, fit, rpn, bc, br, bi))
    x0 = g.token_to_id["x0"]
    h = torch.empty(B1, dtype=torch.int64, device=DEV)
    vp = torch.empty(B1, dtype=torch.int32, device=DEV)
    cases["compute_population_hashes (1M x 64)"] = lambda m: (
        lambda: m.compute_population_hashes(P1, h, vp, 0, x0, 3))
    cases["fitness_sharing_penalty (1M, 4 islands)"] = lambda m: (
        lambda: m.fitness_sharing_penalty(P1, 4, B1 // 4, 2, 8))

    # evaluators and optimisers
    Bf, Df = 1 << 16, 1024
    popf = tl.synthetic.random_programs(g, Bf, 3, 40, 40, rng, max_consts=6)
    cf = T(rng.uniform(-2, 2, (Bf, 6)).astype(np.float32))
    Xf = T(rng.uniform(-2, 2, (3, Df)).astype(np.float32))
    yf = T(np.sin(rng.uniform(-2, 2, Df)).astype(np.float32))
    rm = torch.empty(Bf, dtype=torch.float32, device=DEV)
    Pf = T(popf)
    cases["eval_rpn_fused (64K x 1024 rows)"] = lambda m: (
        lambda: m.eval_rpn_fused(Pf, Xf, cf, yf, rm, *ids, tl.PI_VAL, tl.E_VAL, 0, 0))
    Be, De = 4096, 100_000
    Xe = T(rng.uniform(-2, 2, (3, De)).astype(np.float32))
    pe = torch.empty((Be, De), dtype=torch.float32, device=DEV)
    se = torch.empty((Be, De), dtype=torch.int32, device=DEV)
    ee = torch.empty((Be, De), dtype=torch.uint8, device=DEV)
    cases["eval_rpn (4096 x 100K rows)"] = lambda m: (
        lambda: m.eval_rpn(Pf[:Be], Xe, cf[:Be], pe, se, ee, *ids, tl.PI_VAL, tl.E_VAL, 0))
    Bp = 2048
    gpos = torch.empty((Bp, 6), dtype=torch.float32, device=DEV)
    gerr = torch.empty(Bp, dtype=torch.float32, device=DEV)
    cases["fused_pso (2048 x 32 particles x 20 steps x 1024 rows)"] = lambda m: (
        lambda: m.fused_pso(Pf[:Bp], cf[:Bp], Xf, yf, gpos, gerr, 32, 20, 0.5, 1.5, 1.5, -25.0,
                            25.0, *ids, math.pi, math.e, 3))
    # the engine's own call in a normal generation: PSO_K_NORMAL = 500 programs, nano_pso's
    # default 20 particles, PSO_STEPS_NORMAL = 40 (gpu/config.py:312-315, gpu/engine.py:2137-2174)
    Bn = 500
    gpos_n = torch.empty((Bn, 6), dtype=torch.float32, device=DEV)
    gerr_n = torch.empty(Bn, dtype=torch.float32, device=DEV)
    cases["fused_pso (500 x 20 particles x 40 steps x 1024 rows)"] = lambda m: (
        lambda: m.fused_pso(Pf[:Bn], cf[:Bn], Xf, yf, gpos_n, gerr_n, 20, 40, 0.5, 1.5, 1.5,
                            -25.0, 25.0, *ids, math.pi, math.e, 3))
    gb = tl.GPUGrammar(num_variables=3, operators=('+', '-', '*', '/'))
    popb = tl.synthetic.random_programs(gb, 64, 5, 39, 40, rng, max_consts=6)
    Pb = T(popb)
    cl = T(rng.uniform(-2, 2, (64, 6)).astype(np.float32))
    clw = cl.clone()
    rml = torch.empty(64, dtype=torch.float32, device=DEV)

    def lb(m):
        def run():
            clw.copy_(cl)
            m.lbfgs_optimize(Pb, clw, Xf, yf, rml, 10, 10, 1e-7, -25.0, 25.0, *gb.scalar_ids(),
                             math.pi, math.e)
        return run
    cases["lbfgs_optimize (64 x 1024 rows, 10 iterations)"] = lb
    ga = tl.GPUGrammar(num_variables=3, operators=tl.ALL_OPERATORS)
    art, vt, li, lv, sids = _tables(ga)
    sargs = [T(a) for a in (art, vt, li, lv)]
    pops = literal_rich(ga, 1 << 16, 64, 5)
    Ps = T(pops)

    def simp(m):
        def run():
            t = Ps.clone()
            m.simplify_batch(t, *sargs, 3, *[int(v) for v in sids])
        return run
    cases["simplify_batch (64K x 64, 3 passes; includes a 32 MB copy)"] = simp

    # one generation
    Bv, Lv, Kv, Dv = 4096, 40, 8, 1024
    popv = tl.synthetic.random_programs(g, Bv, 2, Lv, Lv, rng, const_prob=0.4, max_consts=Kv)
    Pv = T(popv)
    cv = T(rng.uniform(-2, 2, (Bv, Kv)).astype(np.float32))
    fv = T(rng.uniform(0.1, 5, Bv).astype(np.float32))
    lv_ = T((popv != 0).sum(1).astype(np.float32))
    e64 = torch.empty(0, dtype=torch.int64, device=DEV)
    bank = T(tl.synthetic.random_programs(g, 64, 2, Lv, Lv, rng, max_consts=Kv))

    def evo(m):
        def run():
            torch.manual_seed(1)
            m.evolve_generation(Pv, cv, fv, e0, Xf, yf, lv_, A, T(a0), T(a1), T(a2), bank, e0,
                                0.1, 0.7, 3, 3, 8, 0.5, 1.5, 1.5, *ids, math.pi, math.e, 4,
                                e64, e64, e64, e64, 99, 5)
        return run
    cases["evolve_generation (4096 x 40, bank, 4 islands, 3 PSO steps x 8)"] = evo
    return cases


@needs_ref
def test_every_export_matches_or_beats_the_reference():
    from warpsymbolic_b200 import rpn_cuda_native as ours
    ref = refext.load("fastmath")
    table = []
    for name, make in _cases().items():
        r = _time(make(ref))
        o = _time(make(ours))
        table.append({"kernel": name, "reference_ms": r, "ours_ms": o, "speedup": r / o})
    tl.write_report("reference_speed_all.json", table)
    # microsecond kernels carry a few microseconds of host wrapper time between the events on
    # both sides: flag only what is clearly slower
    slow = [t for t in table if t["speedup"] < 0.8]
    assert not slow, slow
