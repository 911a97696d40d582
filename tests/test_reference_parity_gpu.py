"""Parity with the reference's OWN kernels (the rpn_cuda_native extension compiled from its
sources with its shipped flags by oracle/build_ref.sh), on identical seeded inputs.

  * eval_rpn drop-in: per-row outputs (prediction bits, stack depth, error byte) identical;
  * eval_rpn_fused drop-in: same invalid/overflow classes, RMSE within 1e-5 relative;
  * eval_fitness, classic policy: the reference's classic evaluate_batch path (eval_rpn +
    torch reductions) within 1e-5 relative, including the C2 workload's programs.

Skipped when the reference build is absent (it needs the reference checkout at build time).
"""
import numpy as np
import pytest
import torch

import refext
import ws_testlib as tl

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(refext.path("fastmath") is None,
                                 reason="reference extension not built (oracle/build_ref.sh)")]
DEV = torch.device("cuda:0") if torch.cuda.is_available() else None


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def same_bits(a, b):
    a = a.cpu().numpy()
    b = b.cpu().numpy()
    both_nan = np.isnan(a) & np.isnan(b)
    return np.array_equal(a[~both_nan].view(np.uint32 if a.dtype == np.float32 else np.uint64),
                          b[~both_nan].view(np.uint32 if b.dtype == np.float32 else np.uint64))


@pytest.mark.parametrize("strict", [0, 1])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_eval_rpn_rows_identical(strict, dtype):
    ref = refext.load("fastmath")
    from warpsymbolic_b200 import rpn_cuda_native as ours
    rng = np.random.default_rng(100 + strict)
    g = tl.GPUGrammar(num_variables=3, operators=tl.ALL_OPERATORS)
    pop, consts = tl.random_population(g, 1500, 48, 6, rng, valid_only=False)
    X = rng.uniform(-4, 4, size=(3, 157)).astype(dtype)
    X[:, :4] = [[0.0, -1.0, 1e-10, 100.0], [2.0, 0.0, -0.0, -50.0], [1.0, 3.0, -2.5, 80.0]]
    c = T(consts.astype(dtype))
    B, D = pop.shape[0], X.shape[1]
    outs = []
    for mod in (ref, ours):
        p = torch.empty((B, D), dtype=c.dtype, device=DEV)
        s = torch.empty((B, D), dtype=torch.int32, device=DEV)
        e = torch.empty((B, D), dtype=torch.uint8, device=DEV)
        mod.eval_rpn(T(pop), T(X), c, p, s, e, *g.scalar_ids(), tl.PI_VAL, tl.E_VAL, strict)
        outs.append((p, s, e))
    torch.cuda.synchronize()
    (rp, rs, re_), (op, os_, oe) = outs
    assert torch.equal(rs, os_)
    assert torch.equal(re_, oe)
    assert same_bits(rp, op)


@pytest.mark.parametrize("V,D", [(1, 1), (1, 17), (2, 32), (3, 33), (4, 333), (2, 1024)])
@pytest.mark.parametrize("strict", [0, 1])
@pytest.mark.parametrize("launch_mode", [0, 1])
def test_eval_rpn_fused_matches_reference(V, D, strict, launch_mode):
    ref = refext.load("fastmath")
    from warpsymbolic_b200 import rpn_cuda_native as ours
    rng = np.random.default_rng(V * 100 + D + 7 * strict)
    g = tl.GPUGrammar(num_variables=V, operators=tl.ALL_OPERATORS)
    pop, consts = tl.random_population(g, 3000, 40, 5, rng, valid_only=False)
    X = rng.uniform(-3, 3, size=(V, D)).astype(np.float32)
    y = rng.standard_normal(D).astype(np.float32)
    r_out = torch.empty(len(pop), dtype=torch.float32, device=DEV)
    o_out = torch.empty_like(r_out)
    args = (T(pop), T(X), T(consts), T(y))
    ref.eval_rpn_fused(*args, r_out, *g.scalar_ids(), tl.PI_VAL, tl.E_VAL, strict, launch_mode)
    ours.eval_rpn_fused(*args, o_out, *g.scalar_ids(), tl.PI_VAL, tl.E_VAL, strict, launch_mode)
    tl.assert_fitness_close(o_out.cpu().numpy(), r_out.cpu().numpy(), rtol=1e-5, atol=1e-7,
                            min_frac=1.0)


@pytest.mark.parametrize("strict", [0, 1])
def test_classic_path_matches_reference(strict):
    ref = refext.load("fastmath")
    rng = np.random.default_rng(200 + strict)
    g = tl.GPUGrammar(num_variables=5, operators=tl.C1_OPERATORS)
    pop, consts = tl.random_population(g, 2000, 64, 8, rng, valid_only=False)
    X = rng.uniform(-3, 3, size=(5, 5000)).astype(np.float32)
    y = rng.standard_normal(5000).astype(np.float32)
    want = refext.classic_rmse(ref, g.scalar_ids(), T(pop), T(X), T(consts), T(y), strict, 1e15)
    from warpsymbolic_b200.cuda_vm import CudaRPNVM
    got = CudaRPNVM(g, DEV).eval_fitness(T(pop), T(X), T(consts), T(y), strict_mode=strict,
                                         policy="classic", loss="rmse", invalid_value=1e15)
    tl.assert_fitness_close(got.cpu().numpy(), want.cpu().numpy(), rtol=1e-5, atol=1e-7,
                            min_frac=1.0)


def test_scale_workload_programs_match_reference():
    """4096 programs of the evaluation-only scale workload on its full 100,000 rows."""
    ref = refext.load("fastmath")
    from warpsymbolic_b200 import synthetic
    from warpsymbolic_b200.cuda_vm import CudaRPNVM
    wl = synthetic.eval_scale_workload(seed=3, n_programs=4096, n_rows=100_000)
    g = wl.grammar
    args = (T(wl.population), T(wl.X), T(wl.constants), T(wl.y))
    want = refext.classic_rmse(ref, g.scalar_ids(), *args, 0, 1e15)
    got = CudaRPNVM(g, DEV).eval_fitness(*args, policy="classic", loss="rmse", invalid_value=1e15)
    tl.assert_fitness_close(got.cpu().numpy(), want.cpu().numpy(), rtol=1e-5, atol=1e-7,
                            min_frac=1.0)
    mse = CudaRPNVM(g, DEV).eval_fitness(*args, policy="classic", loss="mse", invalid_value=1e15)
    v = want.cpu().numpy() < 1e6
    np.testing.assert_allclose(mse.cpu().numpy()[v], want.cpu().numpy()[v].astype(np.float64) ** 2,
                               rtol=3e-5)
