"""One-launch loss and gradient (ws_loss_grad) and the per-program L-BFGS (ws_lbfgs_adjoint) on
the GPU, against the CPU oracle's loss mode and against torch.optim.LBFGS (the optimiser of the
reference's constant-fitting fallback) driven by that oracle, one program at a time."""
import math

import numpy as np
import pytest
import torch

import ws_testlib as tl
from test_constfit_oracle import (SMOOTH_OPS, linear_programs, smooth_case, tmap,
                                  torch_lbfgs_checker)

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0") if torch.cuda.is_available() else None
O = tl.oracle


def T(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a)).to(DEV)
    return t if dtype is None else t.to(dtype)


def cf():
    from warpsymbolic_b200 import constfit
    return constfit


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("shape", [(24, 96), (3, 50_000)])  # one row range / split rows
def test_loss_grad_matches_oracle(dtype, shape):
    B, D = shape
    g, pop, consts, X, y = smooth_case(7, B=B, D=D)
    consts, X, y = consts.astype(dtype), X.astype(dtype), y.astype(dtype)
    loss, grad = cf().loss_grad(T(pop), T(X), T(consts), T(y), g.scalar_ids())
    loss, grad = loss.cpu().numpy(), grad.cpu().numpy().astype(np.float64)
    ol, og, absg = O.loss_grad(tmap(g), pop, X, consts, y)
    fin = np.isfinite(ol)
    assert (np.isfinite(loss) == fin).all()
    # float32 runs the GPU's fast single-precision transcendentals, the oracle libm
    rtol = 1e-11 if dtype == np.float64 else 2e-4
    np.testing.assert_allclose(loss[fin], ol[fin], rtol=rtol, atol=0)
    gtol = (1e-9 if dtype == np.float64 else 2e-3) * (absg + 1e-12)
    assert (np.abs(grad[fin] - og[fin]) <= gtol[fin] + 1e-300).all()


def test_loss_grad_deterministic_active_and_invalid():
    g, pop, consts, X, y = smooth_case(8, B=64, D=4096)
    pop[5, :] = 0
    pop[5, 0] = g.token_to_id['+']  # no result: infinite loss, zero gradient
    P, Xd, cd, yd = T(pop), T(X), T(consts), T(y)
    l1, g1 = cf().loss_grad(P, Xd, cd, yd, g.scalar_ids())
    l2, g2 = cf().loss_grad(P, Xd, cd, yd, g.scalar_ids())
    assert torch.equal(l1, l2) and torch.equal(g1, g2)
    assert math.isinf(float(l1[5])) and bool((g1[5] == 0).all())
    act = torch.zeros(64, dtype=torch.int32, device=DEV)
    act[::3] = 1
    from warpsymbolic_b200 import _native as N
    from warpsymbolic_b200._tensors import ptr, stream_of, workspace
    import ctypes as C
    loss = torch.full((64,), -7.0, dtype=torch.float64, device=DEV)
    grad = torch.full(consts.shape, -7.0, dtype=torch.float64, device=DEV)
    need = C.c_size_t(0)
    N.check(N.lib().ws_loss_grad_workspace_bytes(N.WS_F64, 64, pop.shape[1], 3, 4096,
                                                 consts.shape[1], C.byref(need)))
    ws = workspace(need.value, DEV)
    m = tmap(g)
    N.check(N.lib().ws_loss_grad(N.WS_F64, ptr(P), 64, pop.shape[1], ptr(Xd), 3, 4096, ptr(cd),
                                 consts.shape[1], ptr(yd), ptr(act), ptr(loss), ptr(grad),
                                 C.byref(m), ptr(ws), ws.numel(), stream_of(Xd)))
    on = act.bool()
    assert torch.equal(loss[on], l1[on]) and torch.equal(grad[on], g1[on])
    assert bool((loss[~on] == -7.0).all()) and bool((grad[~on] == -7.0).all())


def test_lbfgs_follows_torch_lbfgs_per_program():
    """float64: each program's run visits the points torch.optim.LBFGS visits with the same
    loss and gradient (the oracle's, on the CPU)."""
    g, pop, consts, X, y = smooth_case(9, B=16, D=256)
    tm = tmap(g)
    out, loss, evals = cf().lbfgs(T(pop), T(X), T(consts), T(y), g.scalar_ids(), max_iter=10,
                                  history_size=5, max_eval=20)
    out, loss, evals = out.cpu().numpy(), loss.cpu().numpy(), evals.cpu().numpy()
    l0, _, _ = O.loss_grad(tm, pop, X, consts, y)
    same = 0
    for b in range(len(pop)):
        if not np.isfinite(l0[b]):
            assert np.array_equal(out[b], consts[b])
            continue
        c_ref, l_ref, calls = torch_lbfgs_checker(tm, pop[b], X, consts[b], y, max_iter=10,
                                                  history=5, max_eval=20)
        assert loss[b] <= l0[b]
        if evals[b] == calls and abs(loss[b] - l_ref) <= 1e-9 * max(abs(l_ref), 1e-12):
            same += 1
        else:  # a rounding-level difference that flipped a line-search decision
            assert loss[b] <= l_ref * (1 + 1e-3) + 1e-12 or loss[b] <= l0[b]
    assert same >= int(0.9 * len(pop)), same


def test_lbfgs_reaches_least_squares():
    g = tl.GPUGrammar(num_variables=3, operators=SMOOTH_OPS)
    pop, design = linear_programs(g)
    rng = np.random.default_rng(3)
    X = rng.uniform(-2, 2, size=(3, 2000))
    y = 1.3 * X[0] - 0.7 * np.sin(X[1]) + 0.2 + 0.01 * rng.standard_normal(2000)
    K = 3
    c0 = np.zeros((len(pop), K))
    out, loss, _ = cf().lbfgs(T(pop), T(X), T(c0), T(y), g.scalar_ids(), max_iter=30,
                              history_size=5)
    loss = loss.cpu().numpy()
    for i in range(len(pop)):
        A = design[i](X)
        coef = np.linalg.lstsq(A, y, rcond=None)[0]
        best = float(((A @ coef - y) ** 2).mean())
        assert loss[i] <= best * (1 + 1e-8) + 1e-14, (i, loss[i], best)


def test_lbfgs_never_worsens_float32_population():
    rng = np.random.default_rng(11)
    g = tl.GPUGrammar(num_variables=3, operators=tl.C1_OPERATORS)
    B, L, K, D = 2048, 40, 8, 1024
    pop = tl.synthetic.random_programs(g, B, 5, L, L, rng, const_prob=0.5, max_consts=K)
    consts = rng.uniform(-3, 3, size=(B, K)).astype(np.float32)
    X = rng.standard_normal((3, D)).astype(np.float32)
    y = (np.sin(X[0]) * 2 + X[1] * X[2]).astype(np.float32)
    P, Xd, cd, yd = T(pop), T(X), T(consts), T(y)
    l0, _ = cf().loss_grad(P, Xd, cd, yd, g.scalar_ids())
    out, loss, evals = cf().lbfgs(P, Xd, cd, yd, g.scalar_ids(), max_iter=10, history_size=5,
                                  max_eval=20)
    l1, _ = cf().loss_grad(P, Xd, out, yd, g.scalar_ids())
    fin = torch.isfinite(l0)
    assert bool((loss[fin] <= l0[fin]).all())
    assert torch.equal(loss[fin], l1[fin])  # the reported loss is the returned point's
    assert bool((evals[fin] >= 1).all()) and int(evals.max()) <= 20 + 25
    improved = (loss[fin] < l0[fin]).float().mean().item()
    assert improved > 0.5, improved
    out2, loss2, evals2 = cf().lbfgs(P, Xd, cd, yd, g.scalar_ids(), max_iter=10,
                                     history_size=5, max_eval=20, sync_every=0)
    assert torch.equal(out, out2) and torch.equal(loss, loss2) and torch.equal(evals, evals2)


def test_optimizer_per_program_accepts_improvements_only():
    from warpsymbolic_b200.evaluation import GPUEvaluator
    from warpsymbolic_b200.optimization import GPUOptimizer
    rng = np.random.default_rng(12)
    g = tl.GPUGrammar(num_variables=2, operators=tl.C1_OPERATORS)
    B, L, K, D = 512, 30, 6, 2048
    pop = tl.synthetic.random_programs(g, B, 5, L, L, rng, const_prob=0.5, max_consts=K)
    consts = rng.uniform(-2, 2, size=(B, K)).astype(np.float32)
    X = rng.uniform(-3, 3, size=(D, 2)).astype(np.float32)
    y = (X[:, 0] ** 2 + 1.5 * np.sin(X[:, 1])).astype(np.float32)
    ev = GPUEvaluator(g, DEV, dtype=torch.float32)
    opt = GPUOptimizer(ev, DEV, dtype=torch.float32)
    P, Xd, cd, yd = T(pop), T(X), T(consts), T(y)
    before = ev.evaluate_batch(P, Xd, yd, cd)
    new_c, errs = opt.lbfgs_optimize_top_k(P, cd, Xd, yd, top_k=B, max_iter=10,
                                           per_program=True, history_size=5)
    assert bool((errs <= before).all())
    after = ev.evaluate_batch(P, Xd, yd, new_c)
    assert torch.equal(after, errs)
    assert float((errs < before).float().mean()) > 0.3


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_loss_grad_long_programs_many_constants(dtype):
    """More than 8 constant slots (shared-memory accumulators) and 120-token programs (a tape too
    long for 4 rows per thread): the other shapes of the kernel."""
    rng = np.random.default_rng(13)
    g = tl.GPUGrammar(num_variables=3, operators=SMOOTH_OPS)
    B, L, K, D = 48, 120, 12, 3000
    pop = tl.synthetic.random_programs(g, B, 40, L, L, rng, const_prob=0.5, max_consts=K)
    consts = rng.uniform(-1, 1, size=(B, K)).astype(dtype)
    X = rng.uniform(-1.5, 1.5, size=(3, D)).astype(dtype)
    y = (np.sin(X[0]) + 0.3 * X[1] * X[2]).astype(dtype)
    loss, grad = cf().loss_grad(T(pop), T(X), T(consts), T(y), g.scalar_ids())
    loss, grad = loss.cpu().numpy(), grad.cpu().numpy().astype(np.float64)
    ol, og, absg = O.loss_grad(tmap(g), pop, X, consts, y)
    fin = np.isfinite(ol) & (ol < 1e30)
    assert fin.sum() > B // 2
    if dtype == np.float64:
        np.testing.assert_allclose(loss[fin], ol[fin], rtol=1e-10, atol=0)
        gtol = 1e-8 * (absg + 1e-12)
        assert (np.abs(grad[fin] - og[fin]) <= gtol[fin] + 1e-300).all()
    else:
        # float32: the GPU's fast single-precision transcendentals against libm, compounded
        # through 120-token chains; nearly every program agrees to 5e-4, none is far off
        rel = np.abs(loss[fin] - ol[fin]) / np.abs(ol[fin])
        assert (rel < 5e-4).mean() > 0.9 and rel.max() < 2e-2, rel.max()
        gerr = np.abs(grad[fin] - og[fin]) / (absg[fin] + 1e-12)
        assert (gerr < 5e-3).mean() > 0.9, (gerr < 5e-3).mean()
    assert (np.abs(og[fin]) > 0).any()
