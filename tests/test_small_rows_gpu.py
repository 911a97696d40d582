"""The small-data-set evaluator (data sets of 1..128 rows, several programs per warp).

`ws_eval_fitness` picks it automatically for 1 <= D <= 128 (schedule 0); explicit schedules
`ws_schedule_count() - 5 + j` run it with 2 << j lanes (8 << j rows) per program.  Checked on the
same inputs against:

  * the row-pass evaluator (schedule 3, 512 rows per pass): identical invalid / overflow classes
    and invalid-row counts, losses within 1e-5 relative (only the order of the sum differs);
  * the CPU oracle in FP64 with correctly rounded operators: exact classes and counts, losses
    to 1e-12;
  * the reference's fused kernel (`rpn_eval_fused_kernel` in its D <= 32 warp mode and block
    mode, the reference extension built from its sources), for the D range where it runs.
"""
import numpy as np
import pytest
import torch

import refext
import ws_testlib as tl

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0") if torch.cuda.is_available() else None
EXACT_OPERATORS = ('+', '-', '*', '/', '%', 'sqrt', 'abs', 'floor', 'ceil', 'sign')
ROWS = [1, 2, 3, 4, 5, 7, 8, 9, 15, 16, 17, 20, 24, 31, 32, 33, 63, 64, 65, 100, 127, 128]


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def small_schedules():
    from warpsymbolic_b200 import _native as N
    n = int(N.lib().ws_schedule_count())
    return {8 << j: n - 5 + j for j in range(5)}  # rows per program -> schedule index


def deep_programs(g, n, rng):
    """Complete binary trees of 32 leaves (63 tokens): the accumulator machine needs 4 spill
    slots for them, the most a 64-token program can need."""
    names = g.active_variables + ['C']
    bins = [o for o in g.operators if g.token_arity[o] == 2]
    pop = np.zeros((n, 64), dtype=np.uint8)
    for i in range(n):
        def build(depth):
            if depth == 0:
                return [names[int(rng.integers(len(names)))]]
            return build(depth - 1) + build(depth - 1) + [bins[int(rng.integers(len(bins)))]]
        toks = build(5)
        pop[i, :len(toks)] = [g.token_to_id[t] for t in toks]
    return pop


def run(g, pop, X, consts, y, schedule=0, **kw):
    from warpsymbolic_b200.cuda_vm import CudaRPNVM
    ninv = torch.empty(len(pop), dtype=torch.int32, device=DEV)
    out = CudaRPNVM(g, DEV).eval_fitness(T(pop), T(X), T(consts), T(y), schedule=schedule,
                                         out_ninvalid=ninv, **kw)
    return out.cpu().numpy(), ninv.cpu().numpy()


@pytest.mark.parametrize("D", ROWS)
@pytest.mark.parametrize("policy,loss,strict", [("classic", "mse", 0), ("fused", "rmse", 0),
                                                ("fused", "rmse", 1), ("classic", "r2", 1)])
def test_small_matches_row_pass_evaluator(D, policy, loss, strict):
    rng = np.random.default_rng(1000 + D + 7 * strict)
    g = tl.GPUGrammar(num_variables=3, operators=tl.ALL_OPERATORS)
    pop, consts = tl.random_population(g, 3000, 48, 6, rng, valid_only=False)
    X = rng.uniform(-3, 3, size=(3, D)).astype(np.float32)
    y = rng.standard_normal(D).astype(np.float32)
    kw = dict(policy=policy, loss=loss, strict_mode=strict)
    got, gn = run(g, pop, X, consts, y, 0, **kw)
    want, wn = run(g, pop, X, consts, y, 3, **kw)
    assert np.array_equal(gn, wn)
    iv = 1e15
    if loss == "r2":  # 1 - R2 = MSE / Var(y); invalid programs (R2 = -iv) map to ~iv
        got, want = 1.0 - got, 1.0 - want
    tl.assert_fitness_close(got, want, rtol=1e-5, atol=1e-6, iv=iv, min_frac=1.0)


@pytest.mark.parametrize("D", [1, 8, 20, 33, 128])
def test_deep_spill_programs(D):
    """Programs that use every spill slot (4 for 64 tokens)."""
    rng = np.random.default_rng(77 + D)
    g = tl.GPUGrammar(num_variables=3, operators=tl.C1_OPERATORS)
    pop = deep_programs(g, 512, rng)
    consts = rng.uniform(-2, 2, size=(512, 6)).astype(np.float32)
    X = rng.uniform(-3, 3, size=(3, D)).astype(np.float32)
    y = rng.standard_normal(D).astype(np.float32)
    got, gn = run(g, pop, X, consts, y, 0, policy="classic", loss="mse")
    want, wn = run(g, pop, X, consts, y, 3, policy="classic", loss="mse")
    assert np.array_equal(gn, wn)
    tl.assert_fitness_close(got, want, rtol=1e-5, atol=1e-6, min_frac=1.0)
    # and against the CPU oracle in FP64 with correctly rounded operators
    g2 = tl.GPUGrammar(num_variables=3, operators=EXACT_OPERATORS)
    pop2 = deep_programs(g2, 512, rng)
    X2, y2, c2 = X.astype(np.float64), y.astype(np.float64), consts.astype(np.float64)
    got2, gn2 = run(g2, pop2, X2, c2, y2, 0, policy="classic", loss="rmse")
    ref2, rn2 = tl.oracle_fitness(g2, pop2, X2, c2, y2, policy="classic", with_ninv=True)
    assert np.array_equal(gn2, rn2)
    tl.assert_fitness_close(got2, ref2, rtol=1e-12, atol=1e-300, iv=1e100, min_frac=1.0)


@pytest.mark.parametrize("D", [1, 5, 16, 20, 64, 100, 128])
@pytest.mark.parametrize("policy", ["fused", "classic"])
@pytest.mark.parametrize("strict", [0, 1])
def test_small_f64_exact_ops_match_oracle(D, policy, strict):
    rng = np.random.default_rng(300 + D + strict)
    g = tl.GPUGrammar(num_variables=3, operators=EXACT_OPERATORS)
    pop, consts = tl.random_population(g, 2000, 48, 6, rng, valid_only=False)
    X = rng.uniform(-3, 3, size=(3, D))
    X[:, :1] = [[0.0], [-1.0], [1e-10]]
    y = X[0] * X[1] + X[2]
    c = consts.astype(np.float64)
    got, gn = run(g, pop, X, c, y, 0, policy=policy, loss="rmse", strict_mode=strict)
    ref, rn = tl.oracle_fitness(g, pop, X, c, y, policy=policy, strict=strict, with_ninv=True)
    assert np.array_equal(gn, rn)
    tl.assert_fitness_close(got, ref, rtol=1e-12, atol=1e-300, iv=1e100, min_frac=1.0)


@pytest.mark.parametrize("D", [1, 8, 9, 20, 32, 40, 64, 100, 128])
def test_every_small_schedule_covering_D(D):
    rng = np.random.default_rng(500 + D)
    g = tl.GPUGrammar(num_variables=2, operators=tl.C1_OPERATORS)
    pop, consts = tl.random_population(g, 1500, 30, 4, rng, valid_only=False)
    X = rng.uniform(-3, 3, size=(2, D)).astype(np.float32)
    y = rng.standard_normal(D).astype(np.float32)
    auto, an = run(g, pop, X, consts, y, 0, policy="classic", loss="mse")
    for rows, sched in small_schedules().items():
        if rows < D:
            with pytest.raises(RuntimeError, match="fewer rows"):
                run(g, pop, X, consts, y, sched, policy="classic", loss="mse")
            continue
        got, gn = run(g, pop, X, consts, y, sched, policy="classic", loss="mse")
        assert np.array_equal(gn, an)
        tl.assert_fitness_close(got, auto, rtol=1e-5, atol=1e-6, min_frac=1.0)


def test_small_schedules_refused_by_batches():
    from warpsymbolic_b200.batch import BatchedFitness, BatchProblem
    rng = np.random.default_rng(5)
    g = tl.GPUGrammar(num_variables=2, operators=tl.C1_OPERATORS)
    pop, consts = tl.random_population(g, 64, 20, 4, rng)
    X = rng.uniform(-3, 3, size=(2, 16)).astype(np.float32)
    y = rng.standard_normal(16).astype(np.float32)
    prob = BatchProblem(T(pop), T(X), T(y), T(consts), g)
    with pytest.raises(RuntimeError, match="one problem per call"):
        BatchedFitness([prob], schedule=list(small_schedules().values())[0])


@pytest.mark.skipif(refext.path("fastmath") is None,
                    reason="reference extension not built (oracle/build_ref.sh)")
@pytest.mark.parametrize("D", [1, 4, 8, 16, 20, 24, 32, 33, 64, 100, 128])
@pytest.mark.parametrize("strict", [0, 1])
def test_small_matches_reference_fused(D, strict):
    ref = refext.load("fastmath")
    from warpsymbolic_b200 import rpn_cuda_native as ours
    rng = np.random.default_rng(900 + D + strict)
    g = tl.GPUGrammar(num_variables=2, operators=tl.ALL_OPERATORS)
    pop, consts = tl.random_population(g, 4096, 30, 5, rng, valid_only=False)
    X = rng.uniform(-3, 3, size=(2, D)).astype(np.float32)
    y = rng.standard_normal(D).astype(np.float32)
    args = (T(pop), T(X), T(consts), T(y))
    r = torch.empty(len(pop), dtype=torch.float32, device=DEV)
    o = torch.empty_like(r)
    mode = 1 if D <= 32 else 0  # the reference autotune's choice (rpn_kernels.cu:2562-2565)
    ref.eval_rpn_fused(*args, r, *g.scalar_ids(), tl.PI_VAL, tl.E_VAL, strict, mode)
    ours.eval_rpn_fused(*args, o, *g.scalar_ids(), tl.PI_VAL, tl.E_VAL, strict, mode)
    tl.assert_fitness_close(o.cpu().numpy(), r.cpu().numpy(), rtol=1e-5, atol=1e-7,
                            min_frac=1.0)
