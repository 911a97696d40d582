"""Seeded synthetic workloads with the shapes and value distributions of the benchmark configs.

No public dataset is used.  Programs are random VALID RPN programs of an exact drawn length,
produced by a stack-depth-constrained sampler (vectorised over programs): at every position
the sampler only offers moves from which the program can still end at depth 1.  Operators are
drawn with the reference's operator weights (config.py:147-153); terminals are the variables
and the constant token `C` (at most `max_consts` per program).  Targets come from random
expression trees evaluated in FP64 with the protected operators.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, Optional, Sequence

import numpy as np

from .grammar import GPUGrammar, PAD_ID

# Reference operator sampling weights (config.py:147-153).
OPERATOR_WEIGHTS: Dict[str, float] = {
    '+': 0.20, '-': 0.20, '*': 0.20, '/': 0.15, 'pow': 0.10, '%': 0.02,
    'sin': 0.10, 'cos': 0.10, 'tan': 0.05, 'log': 0.08, 'exp': 0.08,
    'fact': 0.08, 'floor': 0.01, 'gamma': 0.08, 'lgamma': 0.08,
    'asin': 0.01, 'acos': 0.01, 'atan': 0.01, 'ceil': 0.005,
    'sign': 0.005, 'sqrt': 0.10, 'abs': 0.05, 'neg': 0.02,
}

# The benchmark op set: {+, -, *, protected /, sin, cos, clamped exp, protected log, sqrt|.|, neg}.
BENCH_OPERATORS = ('+', '-', '*', '/', 'sin', 'cos', 'log', 'exp', 'sqrt')


def random_programs(grammar: GPUGrammar, n: int, len_low: int, len_high: int, L: int,
                    rng: np.random.Generator, const_prob: float = 0.3, max_consts: int = 8,
                    cat_weights=(0.45, 0.15, 0.40), use_literals: bool = False) -> np.ndarray:
    """[n, L] uint8 valid RPN programs, lengths ~ U{len_low..len_high} (<= L), PAD-filled."""
    assert 1 <= len_low <= len_high <= L
    lens = rng.integers(len_low, len_high + 1, size=n)
    pop = np.full((n, L), PAD_ID, dtype=np.uint8)
    un = [op for op in grammar.operators if grammar.token_arity[op] == 1]
    bi = [op for op in grammar.operators if grammar.token_arity[op] == 2]
    un_ids = np.array([grammar.token_to_id[o] for o in un], dtype=np.uint8)
    bi_ids = np.array([grammar.token_to_id[o] for o in bi], dtype=np.uint8)
    un_w = np.array([OPERATOR_WEIGHTS.get(o, 0.05) for o in un], dtype=np.float64)
    bi_w = np.array([OPERATOR_WEIGHTS.get(o, 0.05) for o in bi], dtype=np.float64)
    un_cdf = np.cumsum(un_w / un_w.sum())
    bi_cdf = np.cumsum(bi_w / bi_w.sum())
    var_ids = np.array([grammar.token_to_id[v] for v in grammar.active_variables], dtype=np.uint8)
    c_id = grammar.token_to_id['C']
    lit_ids = np.array([grammar.token_to_id[t] for t in ('0', '1', '2', '3', '4', '5', '6', '10',
                                                         'pi', 'e')], dtype=np.uint8)
    depth = np.zeros(n, dtype=np.int64)
    nconst = np.zeros(n, dtype=np.int64)
    wt, wu, wb = cat_weights
    for t in range(L):
        active = t < lens
        if not active.any():
            break
        r_after = lens - t - 1
        can_push = active & (r_after >= depth)
        can_un = active & (depth >= 1) & (r_after >= depth - 1) & (len(un_ids) > 0)
        can_bi = active & (depth >= 2)
        w = np.stack([wt * can_push, wu * can_un, wb * can_bi], axis=1).astype(np.float64)
        tot = w.sum(axis=1)
        tot[tot == 0] = 1.0
        u = rng.random(n) * tot
        cat = np.where(u < w[:, 0], 0, np.where(u < w[:, 0] + w[:, 1], 1, 2))
        tok = np.zeros(n, dtype=np.uint8)
        # terminals
        m0 = active & (cat == 0)
        k0 = int(m0.sum())
        if k0:
            pick_c = (rng.random(k0) < const_prob) & (nconst[m0] < max_consts)
            vars_ = var_ids[rng.integers(0, len(var_ids), size=k0)]
            term = np.where(pick_c, np.uint8(c_id), vars_)
            if use_literals:
                lit = rng.random(k0) < 0.1
                term = np.where(lit & ~pick_c, lit_ids[rng.integers(0, len(lit_ids), size=k0)], term)
            tok[m0] = term
            nconst[m0] += pick_c
            depth[m0] += 1
        m1 = active & (cat == 1)
        k1 = int(m1.sum())
        if k1:
            tok[m1] = un_ids[np.searchsorted(un_cdf, rng.random(k1), side='right').clip(0, len(un_ids) - 1)]
        m2 = active & (cat == 2)
        k2 = int(m2.sum())
        if k2:
            tok[m2] = bi_ids[np.searchsorted(bi_cdf, rng.random(k2), side='right').clip(0, len(bi_ids) - 1)]
            depth[m2] -= 1
        pop[active, t] = tok[active]
    return pop


# ---- targets ------------------------------------------------------------------------------
def _p_div(a, b):
    with np.errstate(all='ignore'):
        return np.where(np.abs(b) < 1e-9, a, a / np.where(np.abs(b) < 1e-9, 1.0, b))


_UNARY = {
    'sin': np.sin, 'cos': np.cos,
    'exp': lambda a: np.exp(np.clip(a, -80.0, 80.0)),
    'log': lambda a: np.log(np.abs(a) + 1e-9),
    'sqrt': lambda a: np.sqrt(np.abs(a)),
    'neg': lambda a: -a,
}
_BINARY = {'+': np.add, '-': np.subtract, '*': np.multiply, '/': _p_div}


def random_tree(rng: np.random.Generator, depth: int, n_vars: int, const_range=(-2.0, 2.0),
                leaf_prob: float = 0.25, unary=('sin', 'cos', 'exp', 'log', 'sqrt', 'neg'),
                binary=('+', '-', '*', '/')):
    """A random expression tree as nested tuples: ('x', i) | ('c', v) | (op, child[, child])."""
    if depth <= 1 or (depth < 4 and rng.random() < leaf_prob):
        if rng.random() < 0.7:
            return ('x', int(rng.integers(0, n_vars)))
        return ('c', float(rng.uniform(*const_range)))
    if rng.random() < 0.3:
        return (str(rng.choice(list(unary))), random_tree(rng, depth - 1, n_vars, const_range,
                                                          leaf_prob, unary, binary))
    return (str(rng.choice(list(binary))),
            random_tree(rng, depth - 1, n_vars, const_range, leaf_prob, unary, binary),
            random_tree(rng, depth - 1, n_vars, const_range, leaf_prob, unary, binary))


def eval_tree(tree, X: np.ndarray) -> np.ndarray:
    """FP64 evaluation of a random_tree over X [V, D] with the protected operators."""
    kind = tree[0]
    if kind == 'x':
        return X[tree[1]].astype(np.float64)
    if kind == 'c':
        return np.full(X.shape[1], tree[1], dtype=np.float64)
    with np.errstate(all='ignore'):
        if len(tree) == 2:
            return _UNARY[kind](eval_tree(tree[1], X))
        return _BINARY[kind](eval_tree(tree[1], X), eval_tree(tree[2], X))


def random_target(rng: np.random.Generator, X: np.ndarray, depth: int, noise_rel: float = 0.0,
                  const_range=(-2.0, 2.0), tries: int = 200):
    """y = tree(X) (+ N(0, (noise_rel*std y)^2)), finite with spread; returns (y f32, tree)."""
    for _ in range(tries):
        tree = random_tree(rng, depth, X.shape[0], const_range)
        y = eval_tree(tree, X)
        if np.all(np.isfinite(y)) and np.std(y) > 1e-3 and np.max(np.abs(y)) < 1e6:
            if noise_rel > 0:
                y = y + rng.normal(0.0, noise_rel * np.std(y), size=y.shape)
            return y.astype(np.float32), tree
    raise RuntimeError("could not draw a finite target")


@dataclass
class EvalWorkload:
    grammar: GPUGrammar
    population: np.ndarray  # [B, L] uint8
    constants: np.ndarray   # [B, K] f32
    X: np.ndarray           # [V, D] f32
    y: np.ndarray           # [D] f32

    def n_tokens(self) -> np.ndarray:
        """Tokens before the first PAD per program (the algorithmic node count)."""
        pad = self.population == PAD_ID
        first = np.where(pad.any(axis=1), pad.argmax(axis=1), self.population.shape[1])
        return first.astype(np.int64)


def eval_scale_workload(seed: int = 0, n_programs: int = 1_048_576, n_rows: int = 100_000,
                        n_vars: int = 5, L: int = 64, len_low: int = 3, len_high: int = 64,
                        K: int = 8, const_range=(-5.0, 5.0), x_range=(-3.0, 3.0),
                        target_depth: int = 5, operators: Optional[Sequence[str]] = None
                        ) -> EvalWorkload:
    """Evaluation-only scale test: random valid programs (lengths U{3..64}), 5 variables, up to
    8 constants U[-5,5], X ~ U[-3,3]^{V x D}, y from a seeded depth-5 random tree."""
    rng = np.random.default_rng(seed)
    g = GPUGrammar(num_variables=n_vars, operators=BENCH_OPERATORS if operators is None else operators)
    pop = random_programs(g, n_programs, len_low, len_high, L, rng, max_consts=K)
    consts = rng.uniform(*const_range, size=(n_programs, K)).astype(np.float32)
    X = rng.uniform(*x_range, size=(n_vars, n_rows)).astype(np.float32)
    y, _ = random_target(rng, X, target_depth)
    return EvalWorkload(g, pop, consts, X, y)


def constopt_workload(seed: int = 0, n_programs: int = 65_536, n_rows: int = 16_384,
                      n_vars: int = 3, L: int = 40, len_low: int = 5, len_high: int = 40,
                      K: int = 8, min_consts: int = 2, const_range=(-3.0, 3.0),
                      target_depth: int = 4, noise_rel: float = 0.01,
                      operators: Optional[Sequence[str]] = None) -> EvalWorkload:
    """Constant-optimisation workload: programs of lengths U{5..40} with 2..8 `C` tokens each,
    K = 8 constant slots U[-3,3], X ~ N(0,1)^{3 x 16,384}, y from a depth-4 tree with constants
    U[-3,3] plus Gaussian noise of sigma = 0.01 * std(y)."""
    rng = np.random.default_rng(seed)
    g = GPUGrammar(num_variables=n_vars, operators=BENCH_OPERATORS if operators is None else operators)
    c_id = g.token_to_id['C']
    pop = random_programs(g, n_programs, len_low, len_high, L, rng, const_prob=0.45, max_consts=K)
    for _ in range(50):  # redraw programs with fewer than min_consts constants
        short = np.nonzero((pop == c_id).sum(axis=1) < min_consts)[0]
        if len(short) == 0:
            break
        pop[short] = random_programs(g, len(short), len_low, len_high, L, rng, const_prob=0.6,
                                     max_consts=K)
    consts = rng.uniform(*const_range, size=(n_programs, K)).astype(np.float32)
    X = rng.standard_normal((n_vars, n_rows)).astype(np.float32)
    y, _ = random_target(rng, X, target_depth, noise_rel=noise_rel, const_range=const_range)
    return EvalWorkload(g, pop, consts, X, y)


@dataclass
class BatchWorkload:
    """Independent regression problems, each an EvalWorkload with its own grammar (variable
    count), rows, population and target."""
    problems: list

    def n_node_evals(self) -> float:
        return float(sum(float(p.n_tokens().sum()) * p.X.shape[1] for p in self.problems))


def batched_workload(seed: int = 0, n_problems: int = 256, programs: int = 2048,
                     rows=(100, 100_000), n_vars=(1, 10), L: int = 64, len_low: int = 3,
                     len_high: int = 64, K: int = 8, const_range=(-2.0, 2.0),
                     x_range=(-4.0, 4.0), depth=(3, 6), noise_rel: float = 0.01,
                     operators: Optional[Sequence[str]] = None) -> BatchWorkload:
    """Batched uneven instances: rows log-uniform in [rows], features uniform in [n_vars],
    X ~ U[x_range], targets from random depth-U{depth} trees with multiplicative relative noise
    y * (1 + noise_rel * N(0, 1)), `programs` random valid programs of lengths U{len_low..len_high}
    per problem."""
    rng = np.random.default_rng(seed)
    ops = BENCH_OPERATORS if operators is None else operators
    lo, hi = np.log10(rows[0]), np.log10(rows[1])
    out = []
    for _ in range(n_problems):
        D = int(np.floor(10.0 ** rng.uniform(lo, hi)))
        V = int(rng.integers(n_vars[0], n_vars[1] + 1))
        g = GPUGrammar(num_variables=V, operators=ops)
        pop = random_programs(g, programs, len_low, len_high, L, rng, max_consts=K)
        consts = rng.uniform(*const_range, size=(programs, K)).astype(np.float32)
        X = rng.uniform(*x_range, size=(V, D)).astype(np.float32)
        y, _ = random_target(rng, X, int(rng.integers(depth[0], depth[1] + 1)))
        y = (y.astype(np.float64) * (1.0 + noise_rel * rng.standard_normal(D))).astype(np.float32)
        out.append(EvalWorkload(g, pop, consts, X, y))
    return BatchWorkload(out)


def serving_stream(seed: int = 0, n_requests: int = 8, rate: float = 20.0,
                   fit_fraction: float = 0.5, rows=(1_000, 200_000), n_vars=(1, 8),
                   population: int = 4096, generations: int = 30, L: int = 64, K: int = 8,
                   x_range=(-3.0, 3.0), depth=(3, 6), noise: float = 0.01,
                   operators: Optional[Sequence[str]] = None) -> list:
    """Serving stream: Poisson arrivals at `rate` per second of fit and evaluate requests; rows
    log-uniform in [rows], features uniform in [n_vars], X ~ U[x_range], targets from random
    depth-U{depth} trees plus N(0, (noise * std y)^2); every request carries `population`
    random programs (the initial population of a fit, or the programs an evaluate scores)."""
    from .serving import Request
    rng = np.random.default_rng(seed)
    ops = BENCH_OPERATORS if operators is None else operators
    lo, hi = np.log10(rows[0]), np.log10(rows[1])
    t = 0.0
    out = []
    for rid in range(n_requests):
        t += float(rng.exponential(1.0 / rate))
        D = int(np.floor(10.0 ** rng.uniform(lo, hi)))
        V = int(rng.integers(n_vars[0], n_vars[1] + 1))
        g = GPUGrammar(num_variables=V, operators=ops)
        pop = random_programs(g, population, 3, L, L, rng, max_consts=K)
        consts = rng.uniform(-2.0, 2.0, size=(population, K)).astype(np.float32)
        X = rng.uniform(*x_range, size=(V, D)).astype(np.float32)
        y, _ = random_target(rng, X, int(rng.integers(depth[0], depth[1] + 1)), noise_rel=noise)
        kind = "fit" if rng.random() < fit_fraction else "evaluate"
        out.append(Request(rid, kind, g, X, y, pop, consts,
                           generations if kind == "fit" else 0, seed * 100_003 + rid, t))
    return out
