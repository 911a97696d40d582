"""CPU pins of the loss-and-gradient oracle (loss mode of oracle/ws_oracle_backward.cpp) and of
the per-program L-BFGS checker (torch.optim.LBFGS with a strong-Wolfe line search, the optimiser
of the reference's constant-fitting fallback, driven by the oracle's loss and gradient):
  - the oracle's loss equals the mean squared error of the classic evaluator where the two
    evaluators' rules coincide, and its gradient matches central finite differences;
  - the L-BFGS checker reaches the least-squares optimum on programs linear in their constants.
"""
import math

import numpy as np
import pytest
import torch

import ws_testlib as tl

O = tl.oracle
SMOOTH_OPS = ('+', '-', '*', 'sin', 'cos', 'exp')


def smooth_case(seed, B=24, L=20, K=4, D=96, V=3):
    rng = np.random.default_rng(seed)
    g = tl.GPUGrammar(num_variables=V, operators=SMOOTH_OPS)
    pop = tl.synthetic.random_programs(g, B, 3, L, L, rng, const_prob=0.5, max_consts=K)
    consts = rng.uniform(-1.5, 1.5, size=(B, K))
    X = rng.uniform(-2, 2, size=(V, D))
    y = np.sin(X[0]) + 0.5 * X[1] * X[2]
    return g, pop, consts, X, y


def tmap(g):
    return tl.N.TokenMap.from_args(*g.scalar_ids(), pi_val=math.pi, e_val=math.e)


def linear_programs(g):
    """Programs linear in their constants: c0*x0 + c1*sin(x1) + c2, c0*x0*x1 + c1, c0 + c1*x2."""
    t = g.token_to_id
    rows = [
        ['C', 'x0', '*', 'C', 'x1', 'sin', '*', '+', 'C', '+'],
        ['C', 'x0', 'x1', '*', '*', 'C', '+'],
        ['C', 'C', 'x2', '*', '+'],
    ]
    L = max(len(r) for r in rows)
    pop = np.zeros((len(rows), L), dtype=np.uint8)
    for i, r in enumerate(rows):
        pop[i, :len(r)] = [t[s] for s in r]
    design = [lambda X: np.stack([X[0], np.sin(X[1]), np.ones_like(X[0])], 1),
              lambda X: np.stack([X[0] * X[1], np.ones_like(X[0])], 1),
              lambda X: np.stack([np.ones_like(X[0]), X[2]], 1)]
    return pop, design


def torch_lbfgs_checker(tm, prog, X, c0, y, max_iter=10, history=5, max_eval=None,
                        grad_clip=1e4):
    """torch.optim.LBFGS(strong Wolfe) on one program, closure = the oracle's loss and
    gradient in float64.  Returns (constants, loss, closure calls)."""
    c = torch.tensor(np.asarray(c0, dtype=np.float64), requires_grad=True)
    opt = torch.optim.LBFGS([c], lr=1.0, max_iter=max_iter, max_eval=max_eval,
                            tolerance_grad=1e-7, tolerance_change=1e-9, history_size=history,
                            line_search_fn="strong_wolfe")
    calls = [0]
    prog2 = prog.reshape(1, -1)

    def closure():
        calls[0] += 1
        opt.zero_grad()
        loss, grad, _ = O.loss_grad(tm, prog2, X, c.detach().numpy().reshape(1, -1), y)
        g = torch.from_numpy(grad[0].copy())
        if grad_clip > 0:
            g = g.clamp(-grad_clip, grad_clip)
        c.grad = g
        return torch.tensor(float(loss[0]), dtype=torch.float64)

    opt.step(closure)
    lf, _, _ = O.loss_grad(tm, prog2, X, c.detach().numpy().reshape(1, -1), y)
    return c.detach().numpy(), float(lf[0]), calls[0]


def test_oracle_loss_is_classic_mse():
    g, pop, consts, X, y = smooth_case(0)
    tm = tmap(g)
    loss, _, _ = O.loss_grad(tm, pop, X, consts, y)
    preds, sp, err = O.eval_rows(tm, pop, X, consts)
    ok = (sp == 1).all(axis=1) & (err == 0).all(axis=1)
    mse = ((preds - y[None, :]) ** 2).mean(axis=1)
    assert ok.sum() >= len(pop) // 2
    np.testing.assert_allclose(loss[ok], mse[ok], rtol=1e-12, atol=0)


def test_oracle_gradient_matches_finite_differences():
    g, pop, consts, X, y = smooth_case(1)
    tm = tmap(g)
    loss, grad, _ = O.loss_grad(tm, pop, X, consts, y)
    h = 1e-6
    checked = 0
    for k in range(consts.shape[1]):
        cp, cm = consts.copy(), consts.copy()
        cp[:, k] += h
        cm[:, k] -= h
        lp, _, _ = O.loss_grad(tm, pop, X, cp, y)
        lm, _, _ = O.loss_grad(tm, pop, X, cm, y)
        fd = (lp - lm) / (2 * h)
        fin = np.isfinite(loss) & (np.abs(loss) < 1e6)
        err = np.abs(grad[fin, k] - fd[fin])
        assert (err <= 1e-5 * np.abs(fd[fin]) + 1e-6 * (1 + loss[fin])).all(), err.max()
        checked += int(fin.sum())
    assert checked > 0


def test_oracle_invalid_program_has_infinite_loss():
    g = tl.GPUGrammar(num_variables=2, operators=SMOOTH_OPS)
    t = g.token_to_id
    pop = np.array([[t['x0'], t['x1'], 0], [t['+'], 0, 0]], dtype=np.uint8)
    X = np.ones((2, 8))
    loss, grad, _ = O.loss_grad(tmap(g), pop, X, np.zeros((2, 1)), np.zeros(8))
    assert np.isinf(loss).all() and (grad == 0).all()


def test_torch_lbfgs_checker_reaches_least_squares():
    g = tl.GPUGrammar(num_variables=3, operators=SMOOTH_OPS)
    pop, design = linear_programs(g)
    rng = np.random.default_rng(3)
    X = rng.uniform(-2, 2, size=(3, 200))
    y = 1.3 * X[0] - 0.7 * np.sin(X[1]) + 0.2 + 0.01 * rng.standard_normal(200)
    tm = tmap(g)
    for i in range(len(pop)):
        A = design[i](X)
        coef = np.linalg.lstsq(A, y, rcond=None)[0]
        best = float(((A @ coef - y) ** 2).mean())
        K = A.shape[1]
        c, lf, calls = torch_lbfgs_checker(tm, pop[i], X, np.zeros(K), y, max_iter=30,
                                           history=5)
        assert lf <= best * (1 + 1e-8) + 1e-14
        assert calls <= 30 * 5 // 4
