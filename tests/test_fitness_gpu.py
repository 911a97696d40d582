"""GPU parity of the evaluation path (eval_rpn, eval_rpn_fused, eval_fitness) through the C ABI.

Checkers: the CPU oracle (oracle/ws_oracle.cpp, C-library math) and the reference's known
answers.  The GPU kernels use the reference's fast-math operator intrinsics, so against the
CPU oracle FP32 values agree to rounding except in ill-conditioned programs; the tests bound
the fraction of such programs and check every class (invalid / overflow / regular) exactly in
FP64.  Bit-level parity with the reference's own kernels is in test_reference_parity_gpu.py.
"""
import json
import math
import os

import numpy as np
import pytest
import torch

import ws_testlib as tl

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
DEV = torch.device("cuda:0") if torch.cuda.is_available() else None


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def vm_for(g):
    from warpsymbolic_b200.cuda_vm import CudaRPNVM
    return CudaRPNVM(g, DEV)


# Operators that are correctly rounded (IEEE) in FP64 on both the GPU and the CPU: with them
# every per-row value is bit-identical, so the whole pipeline must agree with the oracle exactly
# (up to the FP64 order of the final sum).
EXACT_OPERATORS = ('+', '-', '*', '/', '%', 'sqrt', 'abs', 'floor', 'ceil', 'sign')


@pytest.mark.parametrize("policy", ["fused", "classic"])
@pytest.mark.parametrize("strict", [0, 1])
def test_fitness_f64_exact_ops_match_oracle(policy, strict):
    rng = np.random.default_rng(60 + strict)
    g = tl.GPUGrammar(num_variables=3, operators=EXACT_OPERATORS)
    pop, consts = tl.random_population(g, 3000, 48, 6, rng, valid_only=False)
    X = rng.uniform(-3, 3, size=(3, 777))
    X[:, :3] = [[0.0, -1.0, 1e-10], [2.0, 0.0, -0.0], [1.0, 3.0, -2.5]]
    y = X[0] * X[1] + X[2]
    vm = vm_for(g)
    ninv = torch.empty(len(pop), dtype=torch.int32, device=DEV)
    got = vm.eval_fitness(T(pop), T(X), T(consts.astype(np.float64)), T(y), strict_mode=strict,
                          policy=policy, loss="rmse", out_ninvalid=ninv).cpu().numpy()
    ref, rninv = tl.oracle_fitness(g, pop, X, consts.astype(np.float64), y, policy=policy,
                                   strict=strict, with_ninv=True)
    assert np.array_equal(ninv.cpu().numpy(), rninv)
    tl.assert_fitness_close(got, ref, rtol=1e-12, atol=1e-300, iv=1e100, min_frac=1.0)


@pytest.mark.parametrize("policy", ["fused", "classic"])
@pytest.mark.parametrize("strict", [0, 1])
def test_fitness_f64_all_ops_match_oracle(policy, strict):
    """All 22 operators: CUDA's FP64 transcendental functions are within ~1-2 ulp of glibc's;
    discontinuous operators (floor, ceil, sign, %, the rounding inside pow) and cancellation
    turn that into larger differences for a few percent of random programs."""
    rng = np.random.default_rng(10 + strict)
    g = tl.GPUGrammar(num_variables=3, operators=tl.ALL_OPERATORS)
    pop, consts = tl.random_population(g, 2000, 40, 6, rng, valid_only=False)
    X = rng.uniform(-3, 3, size=(3, 333))
    y = np.sin(X[0]) * X[1] + X[2] ** 2
    vm = vm_for(g)
    got = vm.eval_fitness(T(pop), T(X), T(consts.astype(np.float64)), T(y), strict_mode=strict,
                          policy=policy, loss="rmse").cpu().numpy()
    ref = tl.oracle_fitness(g, pop, X, consts.astype(np.float64), y, policy=policy, strict=strict)
    tl.assert_fitness_close(got, ref, rtol=1e-6, atol=1e-12, iv=1e100, min_frac=0.95)


@pytest.mark.parametrize("loss", ["rmse", "mse", "r2", "sse"])
def test_fitness_f32_matches_oracle(loss):
    rng = np.random.default_rng(20)
    g = tl.GPUGrammar(num_variables=2, operators=tl.C1_OPERATORS)
    pop, consts = tl.random_population(g, 4000, 30, 4, rng, valid_only=False)
    X = rng.uniform(-3, 3, size=(2, 1024)).astype(np.float32)
    y = (X[0] ** 2 + 1.5 * np.sin(X[1])).astype(np.float32)
    vm = vm_for(g)
    got = vm.eval_fitness(T(pop), T(X), T(consts), T(y), policy="classic", loss=loss).cpu().numpy()
    ref = tl.oracle_fitness(g, pop, X, consts, y, policy="classic", loss=loss)
    if loss == "r2":
        got, ref = 1.0 - got, 1.0 - ref  # regular values near 0 for good fits: compare 1-R2
    # fast-math intrinsics (as in the reference build) vs the C library: ~1e-4 relative on a
    # few percent of random programs (exp/log/sin of large arguments); exact parity is checked
    # against the reference's own kernels in test_reference_parity_gpu.py
    tl.assert_fitness_close(got, ref, rtol=1e-3, atol=1e-6, min_frac=0.97)


def test_known_answer_rmse_sqrt_7_5():
    """tests/gpu/test_new_bugs_v3.py:461-490: program x0, x=[1,2,3,4], y=2x -> sqrt(7.5)."""
    kat = json.load(open(os.path.join(HERE, "golden", "kats.json")))["rmse_sqrt_7_5"]
    from warpsymbolic_b200.evaluation import GPUEvaluator
    g = tl.GPUGrammar(num_variables=1)
    ev = GPUEvaluator(g, DEV, dtype=torch.float64)
    pop = torch.tensor([g.encode(kat["program"], kat["L"])], dtype=torch.uint8, device=DEV)
    x = torch.tensor(kat["x"], dtype=torch.float64, device=DEV)
    y = torch.tensor(kat["y"], dtype=torch.float64, device=DEV)
    c = torch.zeros(1, kat["K"], dtype=torch.float64, device=DEV)
    r = ev.evaluate_batch(pop, x, y, c)
    assert round(float(r[0]) - kat["expected_rmse"], kat["places"]) == 0
    assert abs(float(r[0]) - math.sqrt(7.5)) < 1e-12


def test_known_answer_x4_passthrough():
    """tests/gpu/test_cuda_eval_modes.py:137-160: with 5 variables, x4 evaluates x4."""
    from warpsymbolic_b200.evaluation import GPUEvaluator
    g = tl.GPUGrammar(num_variables=5)
    ev = GPUEvaluator(g, DEV, dtype=torch.float32)
    pop = torch.full((16, 64), 0, dtype=torch.uint8, device=DEV)
    pop[:, 0] = g.token_to_id["x4"]
    x = torch.randn(5, 41, dtype=torch.float32, device=DEV)
    y = x[4].clone()
    r = ev.evaluate_batch(pop, x, y, torch.empty(16, 0, device=DEV))
    assert torch.allclose(r, torch.zeros_like(r), atol=1e-7, rtol=0)


@pytest.mark.parametrize("samples", [1, 17, 32, 33, 200, 1024])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("strict", [0, 1])
def test_mode_agreement_programs(samples, dtype, strict):
    """tests/gpu/test_cuda_eval_modes.py:51-132: fused-kernel semantics == classic semantics on
    x, x*x, C+x, log x, exp x over linspace(-2, 100) with y = 0; and both equal the oracle."""
    g = tl.GPUGrammar(num_variables=1)
    progs = [["x0"], ["x0", "x0", "*"], ["C", "x0", "+"], ["x0", "log"], ["x0", "exp"]]
    B = 64
    pop = np.array([g.encode(progs[i % 5], 128) for i in range(B)], np.uint8)
    x = np.linspace(-2.0, 100.0, samples).reshape(1, -1)
    npdt = np.float32 if dtype == torch.float32 else np.float64
    x = x.astype(npdt)
    y = np.zeros(samples, npdt)
    c = np.random.default_rng(3).standard_normal((B, 8)).astype(npdt)
    from warpsymbolic_b200.evaluation import GPUEvaluator
    ev = GPUEvaluator(g, DEV, dtype=dtype)
    vm = ev.vm
    fused = vm.eval_fitness(T(pop), T(x), T(c), T(y), strict_mode=strict, policy="fused").cpu().numpy()
    classic = vm.eval_fitness(T(pop), T(x), T(c), T(y), strict_mode=strict, policy="classic",
                              invalid_value=ev.INF_VAL).cpu().numpy()
    thr = 1e14 if dtype == torch.float32 else 1e99
    assert np.array_equal(fused >= thr, classic >= thr)
    v = fused < thr
    tol = 2e-5 if dtype == torch.float32 else 1e-10
    assert np.allclose(fused[v], classic[v], rtol=tol, atol=tol)
    ref = tl.oracle.fused_rmse(tl.token_map(g), pop, x, c, y, strict=strict)
    assert np.array_equal(fused >= thr, ref >= thr)
    assert np.allclose(fused[v], ref[v], rtol=1e-4 if dtype == torch.float32 else 1e-10, atol=tol)


@pytest.mark.parametrize("B,L,V,D", [(1, 1, 1, 1), (7, 2, 1, 3), (33, 64, 5, 255), (100, 64, 5, 257),
                                     (5, 256, 12, 1000), (3, 30, 2, 70001), (2048, 64, 10, 100),
                                     (64, 40, 0, 50)])
def test_fitness_edge_shapes(B, L, V, D):
    rng = np.random.default_rng(B * 1000 + D)
    g = tl.GPUGrammar(num_variables=max(V, 1), operators=EXACT_OPERATORS)
    if V == 0:
        # programs of constants/literals only, x has zero rows
        pop = np.zeros((B, L), np.uint8)
        for i in range(B):
            pop[i, :3] = [g.token_to_id["C"], g.token_to_id["pi"], g.token_to_id["*"]]
        X = np.zeros((0, D), np.float64)
    else:
        pop, _ = tl.random_population(g, B, L, 3, rng, valid_only=False)
        X = rng.uniform(-3, 3, size=(V, D))
    consts = rng.uniform(-2, 2, size=(B, 3))
    y = rng.standard_normal(D)
    from warpsymbolic_b200.cuda_vm import CudaRPNVM
    vm = CudaRPNVM(g, DEV)
    vm.num_vars = V
    import ctypes
    from warpsymbolic_b200 import _native as N
    vm._tmap = N.TokenMap.from_args(*g.scalar_ids(), pi_val=tl.PI_VAL, e_val=tl.E_VAL)
    got = vm.eval_fitness(T(pop), T(X), T(consts), T(y), policy="classic", loss="mse").cpu().numpy()
    m = tl.token_map(g)
    ref = tl.oracle.fitness(m, pop, X, consts, y, policy="classic", loss="mse")
    tl.assert_fitness_close(got, ref, rtol=1e-12, atol=1e-300, iv=1e100, min_frac=1.0)


def test_batch_invariance_and_determinism():
    """A program's loss does not depend on the batch it is evaluated in, nor on the run."""
    rng = np.random.default_rng(5)
    g = tl.GPUGrammar(num_variables=3, operators=tl.C1_OPERATORS)
    pop, consts = tl.random_population(g, 3000, 48, 6, rng, valid_only=True)
    X = rng.uniform(-3, 3, size=(3, 50000)).astype(np.float32)
    y = (X[0] * X[1] - np.cos(X[2])).astype(np.float32)
    vm = vm_for(g)
    full = vm.eval_fitness(T(pop), T(X), T(consts), T(y), policy="classic").cpu().numpy()
    again = vm.eval_fitness(T(pop), T(X), T(consts), T(y), policy="classic").cpu().numpy()
    assert np.array_equal(full.view(np.uint32), again.view(np.uint32))
    for i in (0, 17, 2999):
        alone = vm.eval_fitness(T(pop[i:i + 1]), T(X), T(consts[i:i + 1]), T(y),
                                policy="classic").cpu().numpy()
        assert alone.view(np.uint32)[0] == full.view(np.uint32)[i]


def test_eval_rpn_dropin_matches_oracle_rows():
    rng = np.random.default_rng(30)
    g = tl.GPUGrammar(num_variables=3, operators=tl.ALL_OPERATORS)
    pop, consts = tl.random_population(g, 700, 40, 5, rng, valid_only=False)
    X = rng.uniform(-3, 3, size=(3, 97))
    from warpsymbolic_b200.cuda_vm import CudaRPNVM
    vm = CudaRPNVM(g, DEV)
    for strict in (0, 1):
        p, s, e = vm.eval(T(pop), T(X), T(consts), strict_mode=strict)
        rp, rs, re_ = tl.oracle.eval_rows(tl.token_map(g), pop, X, consts, strict=strict)
        # FP64 transcendental functions differ by ~1 ulp between CUDA and glibc; discontinuous
        # operators occasionally turn that into a different error flag or value
        assert (s.cpu().numpy() == rs).mean() > 0.995
        assert (e.cpu().numpy() == re_).mean() > 0.995
        pc = p.cpu().numpy()
        ok = (rs == 1) & (re_ == 0) & np.isfinite(rp)
        close = np.isclose(pc[ok], rp[ok], rtol=1e-9, atol=1e-12)
        assert close.mean() > 0.99


def test_eval_rpn_fused_dropin_errors_and_values():
    from warpsymbolic_b200 import rpn_cuda_native as R
    g = tl.GPUGrammar(num_variables=2, operators=tl.C1_OPERATORS)
    rng = np.random.default_rng(40)
    pop, consts = tl.random_population(g, 300, 30, 4, rng, valid_only=False)
    X = rng.uniform(-3, 3, size=(2, 300)).astype(np.float32)
    y = (X[0] ** 2 + 1.5 * np.sin(X[1])).astype(np.float32)
    out = torch.empty(300, dtype=torch.float32, device=DEV)
    ids = g.scalar_ids()
    R.eval_rpn_fused(T(pop), T(X), T(consts), T(y), out, *ids, tl.PI_VAL, tl.E_VAL)
    ref = tl.oracle.fused_rmse(tl.token_map(g), pop, X, consts, y)
    tl.assert_fitness_close(out.cpu().numpy(), ref, rtol=1e-3, min_frac=0.97)
    with pytest.raises(RuntimeError, match="supports 1..1024 samples"):
        Xb = torch.zeros(2, 1025, device=DEV)
        R.eval_rpn_fused(T(pop), Xb, T(consts), torch.zeros(1025, device=DEV), out, *ids,
                         tl.PI_VAL, tl.E_VAL)
    with pytest.raises(RuntimeError, match="must be a CUDA tensor"):
        R.eval_rpn_fused(torch.from_numpy(pop), T(X), T(consts), T(y), out, *ids, tl.PI_VAL, tl.E_VAL)


def test_validate_strict_counts_match_oracle():
    from warpsymbolic_b200.evaluation import GPUEvaluator
    rng = np.random.default_rng(50)
    g = tl.GPUGrammar(num_variables=2, operators=tl.ALL_OPERATORS)
    pop, consts = tl.random_population(g, 500, 32, 4, rng, valid_only=False)
    X = rng.uniform(-3, 3, size=(2, 211))
    y = X[0] - X[1]
    ev = GPUEvaluator(g, DEV, dtype=torch.float64)
    res = ev.validate_strict(T(pop), T(X), T(y), T(consts))
    _, rninv = tl.oracle_fitness(g, pop, X, consts, y, policy="classic", strict=1, with_ninv=True)
    assert (res["n_errors"].cpu().numpy() == rninv).mean() > 0.998
    assert res["n_total"] == 211
