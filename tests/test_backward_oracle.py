"""The adjoint oracle (oracle/ws_oracle_backward.cpp) pinned on CPU: known answers for the
reference's rules (backward_kernels.cu:13-281), central finite differences and torch autograd
on differentiable programs.  The reference's own test of this path asserts nothing
(tests/gpu/test_native_autograd.py), so calculus is the pin."""
import numpy as np
import pytest
import torch

import ws_testlib as tl

O = tl.oracle
DIFF_OPS = ('+', '-', '*', '/', 'sin', 'cos', 'log', 'exp')


def _bwd(g, prog_tokens, K, consts, X, gout=None, L=None):
    L = L or max(len(p) for p in prog_tokens)
    pop = np.array([g.encode(p, L) for p in prog_tokens], dtype=np.uint8)
    B, D = len(prog_tokens), X.shape[1]
    c = np.asarray(consts, dtype=X.dtype).reshape(B, K)
    gout = np.ones((B, D), dtype=X.dtype) if gout is None else gout
    return O.backward(tl.token_map(g), pop, X, c, gout)


def test_known_answers_of_the_reference_rules():
    g = tl.GPUGrammar(num_variables=1, operators=tl.ALL_OPERATORS)
    X = np.array([[0.5, 1.5, -2.0]])
    x = X[0]
    c = 0.7
    cases = [
        (["C", "x0", "*"], 1, [c], np.sum(x)),                 # d(C*x)/dC
        (["C", "sin"], 1, [c], 3 * np.cos(c)),
        (["C", "cos"], 1, [c], -3 * np.sin(c)),
        (["C", "exp"], 1, [c], 3 * np.exp(c)),
        (["C", "log"], 1, [c], 3 / c),
        (["C", "sqrt"], 1, [c], 3 * 0.5 / np.sqrt(c)),
        (["C", "neg"], 1, [c], -3.0),
        (["C", "C", "+"], 1, [c], 6.0),                          # both C tokens use slot 0
        (["C", "C", "-"], 2, [c, 0.2], None),                    # checked per slot below
        (["C", "tan"], 1, [c], 0.0),                             # no adjoint through tan
        (["C", "abs"], 1, [c], 0.0),                             # ... nor abs
        (["C", "x0", "%"], 1, [c], 0.0),                         # ... nor %
        (["C", "floor"], 1, [c], 0.0),                           # forward 0, no adjoint
        (["C", "x0"], 1, [c], 0.0),                              # two results: skipped
        (["C", "+"], 1, [c], 3.0),                               # stops at '+': root is C
        (["C", "x0", "/"], 1, [c], np.sum(1 / x)),
        (["x0", "C", "/"], 1, [c], np.sum(-x / c ** 2)),
        (["C", "x0", "pow"], 1, [c], np.sum(x * c ** (x - 1))),
        (["x0", "C", "pow"], 1, [c], np.sum(np.where(x > 0, np.abs(x) ** c * np.log(np.abs(x)),
                                                     0.0))),
    ]
    for prog, K, consts, want in cases:
        grad, _ = _bwd(g, [prog], K, consts, X)
        if want is None:
            assert grad[0].tolist() == [3.0, -3.0], prog
        else:
            assert grad[0, 0] == pytest.approx(want, rel=1e-12, abs=1e-12), prog


def test_stack_limit_and_slot_clamp():
    g = tl.GPUGrammar(num_variables=1, operators=tl.C1_OPERATORS)
    X = np.array([[1.0, 2.0]])
    # 33 pushes: the 33rd is dropped (stack of 32), 31 additions leave one value -> valid;
    # the dropped C (slot clamped to K-1 = 1) receives nothing.
    prog = ["C"] * 32 + ["C"] + ["+"] * 31
    grad, _ = _bwd(g, [prog], 2, [0.1, 0.2], X)
    assert grad[0].tolist() == [2.0, 31 * 2.0]


def _diff_population(seed, B, L, K, V):
    rng = np.random.default_rng(seed)
    g = tl.GPUGrammar(num_variables=V, operators=DIFF_OPS)
    pop = tl.synthetic.random_programs(g, B, 3, L, L, rng, max_consts=K)
    consts = rng.uniform(-1.5, 1.5, size=(B, K))
    X = rng.uniform(-2, 2, size=(V, 64))
    gout = rng.standard_normal((B, 64))
    return g, pop, consts, X, gout


def test_central_differences():
    """adjoint == d/dC sum_d g_d * pred_d, with Richardson-extrapolated central differences
    (h = 1e-3 and 5e-4) of the oracle's own forward evaluator, FP64."""
    B, L, K, V = 300, 20, 4, 2
    g, pop, consts, X, gout = _diff_population(1, B, L, K, V)
    tm = tl.token_map(g)
    grad, absg = O.backward(tm, pop, X, consts, gout)

    def S(c):
        preds, sp, err = O.eval_rows(tm, pop, X, c)
        return (np.where((sp == 1) & (err == 0), preds, 0.0) * gout).sum(axis=1)

    def fd(h):
        out = np.zeros((B, K))
        for k in range(K):
            cp, cm = consts.copy(), consts.copy()
            cp[:, k] += h
            cm[:, k] -= h
            out[:, k] = (S(cp) - S(cm)) / (2 * h)
        return out

    f1, f2 = fd(1e-3), fd(5e-4)
    rich = (4 * f2 - f1) / 3
    used = absg > 0
    assert np.array_equal(grad[~used], np.zeros((~used).sum()))
    # pairs where the differences converge (steep exp / near-zero divisors excluded) and no exp
    # argument saturates at +-80 (there the reference's rule passes e^80 * adj, while the
    # clamped forward is flat); the Richardson correction |f1 - f2| bounds the remaining
    # truncation error
    smooth = (np.abs(f1 - f2) <= 1e-2 * np.abs(f2) + 1e-9) & (absg < 1e20)
    ok = np.abs(grad - rich) <= np.maximum(np.abs(f1 - f2), 1e-7 * np.abs(rich) + 1e-9)
    sel = used & smooth
    assert sel.sum() > 0.9 * used.sum()
    assert ok[sel].all(), np.argwhere(sel & ~ok)[:5]


def _torch_forward(g, prog, c, X):
    """Differentiable torch restatement of the forward rules for the DIFF_OPS programs."""
    ids = {v: k for k, v in g.token_to_id.items()}
    stack, ci = [], 0
    K = c.shape[0]
    for t in prog:
        if t == 0:
            break
        name = ids[int(t)]
        if name.startswith("x"):
            stack.append(X[int(name[1:])])
        elif name == "C":
            stack.append(c[min(ci, K - 1)].expand(X.shape[1]))
            ci += 1
        elif name in ("+", "-", "*", "/"):
            b_, a_ = stack.pop(), stack.pop()
            if name == "+":
                stack.append(a_ + b_)
            elif name == "-":
                stack.append(a_ - b_)
            elif name == "*":
                stack.append(a_ * b_)
            else:
                stack.append(torch.where(b_.abs() < 1e-9, a_, a_ / b_))
        else:
            a_ = stack.pop()
            f = {"sin": torch.sin, "cos": torch.cos, "neg": torch.neg,
                 "log": lambda v: torch.log(v.abs() + 1e-9),
                 "exp": lambda v: torch.exp(v.clamp(-80, 80))}[name]
            stack.append(f(a_))
    assert len(stack) == 1
    return stack[0]


def test_torch_autograd():
    B, L, K, V = 200, 24, 4, 3
    g, pop, consts, X, gout = _diff_population(2, B, L, K, V)
    grad, absg = O.backward(tl.token_map(g), pop, X, consts, gout)
    Xt = torch.from_numpy(X)
    agree = 0
    for b in range(B):
        c = torch.tensor(consts[b], requires_grad=True)
        s = (_torch_forward(g, pop[b], c, Xt) * torch.from_numpy(gout[b])).sum()
        gt = torch.autograd.grad(s, c, allow_unused=True)[0] if s.requires_grad else None
        gt = np.zeros(K) if gt is None else gt.numpy()
        # torch differentiates log(|a| + 1e-9) exactly (sign(a) / (|a| + 1e-9)); the
        # reference's rule is 1 / a: they differ by the 1e-9 shift, relatively ~1e-9 / |a|
        agree += np.all(np.abs(gt - grad[b]) <= 1e-6 * (absg[b] + np.abs(gt)) + 1e-300)
    assert agree >= 0.98 * B
