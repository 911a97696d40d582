"""Particle swarm: pso_update, pso_update_bests and the fused PSO loop.

CPU (oracle/ws_oracle_pso.cpp): the update formula against numpy, the bests' tie rule on hand
cases.  GPU: bit-exact against the reference extension's own kernels on identical inputs and
seeds; the fused loop's reported error against the oracle's PSO fitness of the reported
constants; the reference's argument checks and messages.
"""
import math

import numpy as np
import pytest
import torch

import refext
import ws_testlib as tl

O = tl.oracle
gpu = pytest.mark.gpu
needs_ref = pytest.mark.skipif(refext.path("fastmath") is None,
                               reason="reference extension not built (oracle/build_ref.sh)")


def _state(seed, B, P, K, dtype):
    rng = np.random.default_rng(seed)
    f = lambda *s: rng.standard_normal(s).astype(dtype)  # noqa: E731
    return (f(B, P, K), f(B, P, K), f(B, P, K), f(B, K), rng.random((B, P, K)).astype(dtype),
            rng.random((B, P, K)).astype(dtype))


def test_oracle_update_formula():
    pos, vel, pb, gb, r1, r2 = _state(1, 3, 5, 4, np.float64)
    p2, v2 = O.pso_update(pos, vel, pb, gb, r1, r2, 0.7, 1.5, 1.3)
    w, c1, c2 = np.float64(np.float32(0.7)), np.float64(np.float32(1.5)), np.float64(np.float32(1.3))
    nv = w * vel + c1 * r1 * (pb - pos) + c2 * r2 * (gb[:, None, :] - pos)
    np.testing.assert_allclose(v2, nv, rtol=1e-15)
    np.testing.assert_allclose(p2, pos + nv, rtol=1e-15)


def test_oracle_bests_tie_rule():
    """Personal bests improve on strictly smaller errors; the swarm minimum is taken over a
    32-lane stride (lane t sees particles t, t+32, ...: the first minimum of the lane), then a
    shuffle-down tree in which a lane takes its partner's value only when strictly smaller, so
    equal minima resolve by the tree's pairing; NaN and >= 1e30 never win; the swarm best
    changes only when strictly better."""
    B, P, K = 4, 40, 2
    cur = np.full((B, P), 5.0)
    cur[0, [2, 33]] = 1.0          # lanes 2 and 1: lane 0 takes lane 2 first (offset 2),
                                   # then keeps it against lane 1 (offset 1): particle 2
    cur[1, [7, 39]] = 1.0          # lanes 7 and 7: particle 7 (first in the lane) wins
    cur[2, :] = np.nan             # nothing improves
    cur[3, 4] = 0.5                # better than the swarm best of 0.75? yes
    pb_err = np.full((B, P), 9.0)
    pb_err[2, :] = 1e30
    cur_pos = np.arange(B * P * K, dtype=np.float64).reshape(B, P, K)
    pb_pos = np.zeros((B, P, K))
    gb_err = np.array([2.0, 2.0, 2.0, 0.75])
    gb_pos = np.full((B, K), -1.0)
    pe, pp, ge, gp = O.pso_update_bests(cur, pb_err, pb_pos, cur_pos, gb_err, gb_pos)
    assert ge.tolist() == [1.0, 1.0, 2.0, 0.5]
    assert gp[0].tolist() == cur_pos[0, 2].tolist()
    assert gp[1].tolist() == cur_pos[1, 7].tolist()
    assert gp[2].tolist() == [-1.0, -1.0]
    assert gp[3].tolist() == cur_pos[3, 4].tolist()
    assert (pe[0] == np.minimum(9.0, cur[0])).all()


def test_oracle_pso_fitness_rules():
    """The fused PSO's fitness on hand cases with exactly representable values: eval_rpn_single's
    domain errors, underflow / leftover values, the constant-slot clamp, the push-drop at depth
    32, unknown tokens (pop one, push 0) and the sequential RMSE (fused_pso_kernels.cu:57-197,
    330-351)."""
    g = tl.GPUGrammar(num_variables=2, operators=tl.ALL_OPERATORS)
    tm = tl.token_map(g)
    L = 64
    X = np.array([[1, 2, 3, 4], [0.5, -1, 0, 2]], dtype=np.float32)
    y = np.array([1, 3, 5, 7], dtype=np.float32)
    inf = np.float32(1e30)
    rms = lambda pred: np.float32(np.sqrt(np.mean((np.asarray(pred, np.float64) - y) ** 2)))  # noqa: E731
    cases = [  # (tokens, constants, expected RMSE)
        (["x0", "C", "*"], [2.0], 1.0),                       # 2 x0 - y = 1 on every row
        (["x0", "x1", "/"], [0.0], inf),                      # x1 = 0 on row 2: |b| < 1e-12
        (["x1", "log"], [0.0], inf),                          # log of <= 1e-12
        (["x1", "sqrt"], [0.0], inf),                         # sqrt of a negative
        (["x0", "sqrt"], [0.0], rms(np.sqrt(X[0]))),
        (["C", "exp"], [81.0], inf),                          # exp above 80: error
        (["C", "exp"], [-81.0], rms([0, 0, 0, 0])),           # exp below -80: 0, no error
        (["+"], [0.0], inf),                                  # underflow
        (["x0", "x1"], [0.0], inf),                           # two values left
        (["C", "C", "+", "x0", "+"], [3.0], rms(6 + X[0])),   # the second C clamps to slot K-1
        (["x0", "2", "pow"], [0.0], rms(X[0] ** 2)),
        (["C", "fact"], [-1.0], inf),                         # fact at a negative integer
        (["C", "fact", "x0", "*"], [3.0], rms(6 * X[0])),
        (["C", "C", "*"], [1e15], inf),                       # finite 1e30 >= 1e29: an error
        (["x0", "1", "asin"], [0.0], inf),                    # asin(1) fine, two values left
        (["C", "x0", "%"], [0.0], rms(np.zeros(4))),          # 0 mod x0 = 0
    ]
    pop = np.array([g.encode(t, L) for t, _, _ in cases], dtype=np.uint8)
    consts = np.array([c for _, c, _ in cases], dtype=np.float32)
    extra = []
    # push-drop: 33 pushes keep 32 values, 31 additions then leave one: 32 x0
    extra.append((g.encode(["x0"] * 33 + ["+"] * 31, L), rms(32 * X[0])))
    # an unknown token pops one value and pushes 0
    row = g.encode(["x0", "x1"], L)
    row[2] = 250
    extra.append((row, inf))                                  # x0 0: two values left
    row = g.encode(["x0"], L)
    row[1] = 250
    extra.append((row, rms(np.zeros(4))))
    pop = np.concatenate([pop, np.array([r for r, _ in extra], dtype=np.uint8)])
    consts = np.concatenate([consts, np.zeros((len(extra), 1), np.float32)])
    want = np.array([e for _, _, e in cases] + [e for _, e in extra], dtype=np.float32)
    got = O.pso_rmse(tm, pop, X, consts, y)
    np.testing.assert_allclose(got, want, rtol=1e-6)


# ---------------------------------------------------------------------------------------------
DEV = torch.device("cuda:0") if torch.cuda.is_available() else None


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


@gpu
@needs_ref
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("B,P,K", [(300, 20, 4), (17, 64, 16), (1000, 3, 1)])
def test_pso_update_bit_exact(dtype, B, P, K):
    ref = refext.load("fastmath")
    from warpsymbolic_b200 import rpn_cuda_native as ours
    pos, vel, pb, gb, r1, r2 = _state(B + P, B, P, K, dtype)
    outs = []
    for mod in (ref, ours):
        p, v = T(pos), T(vel)
        mod.pso_update(p, v, T(pb), T(gb), T(r1), T(r2), 0.6123, 1.49445, 1.3)
        outs.append((p.cpu().numpy(), v.cpu().numpy()))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    op, ov = O.pso_update(pos, vel, pb, gb, r1, r2, 0.6123, 1.49445, 1.3)
    tol = 1e-5 if dtype == np.float32 else 1e-13
    np.testing.assert_allclose(outs[1][1], ov, rtol=tol, atol=tol)


@gpu
@needs_ref
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("B,P,K", [(500, 20, 4), (64, 100, 3), (2000, 7, 0)])
def test_pso_update_bests_bit_exact(dtype, B, P, K):
    ref = refext.load("fastmath")
    from warpsymbolic_b200 import rpn_cuda_native as ours
    rng = np.random.default_rng(B)
    cur = np.round(rng.random((B, P)) * 8).astype(dtype)   # many ties
    cur[rng.random((B, P)) < 0.05] = np.nan
    pbe = np.round(rng.random((B, P)) * 8 + 1).astype(dtype)
    pbe[::7] = 1e30
    cur_pos = rng.standard_normal((B, P, K)).astype(dtype)
    pb_pos = rng.standard_normal((B, P, K)).astype(dtype)
    gbe = np.round(rng.random(B) * 4).astype(dtype)
    gb_pos = rng.standard_normal((B, K)).astype(dtype)
    outs = []
    for mod in (ref, ours):
        a = [T(pbe), T(pb_pos), T(gbe), T(gb_pos)]
        mod.pso_update_bests(T(cur), a[0], a[1], T(cur_pos), a[2], a[3])
        outs.append([t.cpu().numpy() for t in a])
    for r, o in zip(*outs):
        assert np.array_equal(r, o, equal_nan=True)
    for w, o in zip(O.pso_update_bests(cur, pbe, pb_pos, cur_pos, gbe, gb_pos), outs[1]):
        assert np.array_equal(w, o, equal_nan=True)


def _fused_case(seed, B, L, K, D, V=2, ops=tl.C1_OPERATORS, valid_only=True):
    rng = np.random.default_rng(seed)
    g = tl.GPUGrammar(num_variables=V, operators=ops)
    pop, consts = tl.random_population(g, B, L, K, rng, valid_only=valid_only)
    X = rng.uniform(-3, 3, size=(V, D)).astype(np.float32)
    y = (X[0] ** 2 + 1.5 * np.sin(X[-1]) + rng.normal(0, 0.01, D)).astype(np.float32)
    return g, pop, consts.astype(np.float32), X, y


def _run_fused(mod, g, pop, consts, X, y, P, steps, seed, w=0.5, c1=1.5, c2=1.5, cmin=-25.0,
               cmax=25.0):
    B, K = consts.shape
    gp = torch.empty((B, K), dtype=torch.float32, device=DEV)
    ge = torch.empty(B, dtype=torch.float32, device=DEV)
    mod.fused_pso(T(pop), T(consts), T(X), T(y), gp, ge, P, steps, w, c1, c2, cmin, cmax,
                  *g.scalar_ids(), math.pi, math.e, seed)
    torch.cuda.synchronize()
    return gp.cpu().numpy(), ge.cpu().numpy()


@gpu
@needs_ref
@pytest.mark.parametrize("B,P,steps,K,D,ops", [
    (700, 20, 20, 4, 200, tl.C1_OPERATORS),   # row split, eight warps per swarm
    (500, 20, 10, 4, 1024, tl.C1_OPERATORS),  # row split, eight warps, four 256-row chunks
    (4500, 32, 4, 8, 300, tl.C1_OPERATORS),   # row split, four warps (beyond seven waves)
    (200, 30, 6, 5, 1, tl.C1_OPERATORS),      # a single row
    (700, 40, 10, 10, 96, tl.C1_OPERATORS),   # above 32 particles: row groups of two warps
    (700, 64, 5, 16, 1024, tl.C1_OPERATORS),
    (4500, 48, 3, 4, 200, tl.C1_OPERATORS),   # two-warp row groups, four warps per swarm
    (700, 7, 12, 3, 333, tl.ALL_OPERATORS),
])
def test_fused_pso_bit_exact(B, P, steps, K, D, ops):
    ref = refext.load("fastmath")
    from warpsymbolic_b200 import rpn_cuda_native as ours
    g, pop, consts, X, y = _fused_case(P + K, B, 30, K, D, ops=ops,
                                       valid_only=ops is tl.C1_OPERATORS)
    seed = 123456789 + P
    rp, re_ = _run_fused(ref, g, pop, consts, X, y, P, steps, seed)
    op, oe = _run_fused(ours, g, pop, consts, X, y, P, steps, seed)
    assert np.array_equal(re_, oe, equal_nan=True), np.nonzero(re_ != oe)[0][:5]
    assert np.array_equal(rp, op, equal_nan=True)
    # the reported error is the fitness of the reported constants (oracle, host libm)
    tm = tl.N.TokenMap.from_args(*g.scalar_ids(), pi_val=math.pi, e_val=math.e)
    fit = O.pso_rmse(tm, pop, X, op, y)
    both_inf = (oe >= 1e29) & (fit >= 1e29)
    close = np.abs(fit - oe) <= 1e-3 * np.abs(oe) + 1e-5
    assert (both_inf | close).mean() > 0.97
    # particle 0 starts at the initial constants: the swarm never ends worse than them
    init_fit = O.pso_rmse(tm, pop, X, consts, y)
    assert ((oe <= init_fit * (1 + 1e-4) + 1e-6) | (init_fit >= 1e29)).mean() > 0.99
    assert (oe < 1e29).mean() > 0.3


@gpu
@needs_ref
@pytest.mark.parametrize("P", [20, 48])
def test_fused_pso_zero_steps(P):
    """No step: the swarm best stays the initial constants with the error sentinel."""
    ref = refext.load("fastmath")
    from warpsymbolic_b200 import rpn_cuda_native as ours
    g, pop, consts, X, y = _fused_case(5, 300, 30, 4, 128)
    rp, re_ = _run_fused(ref, g, pop, consts, X, y, P, 0, 77)
    op, oe = _run_fused(ours, g, pop, consts, X, y, P, 0, 77)
    assert np.array_equal(re_, oe, equal_nan=True)
    assert np.array_equal(rp, op, equal_nan=True)
    assert np.array_equal(op, consts) and (oe == np.float32(1e30)).all()


@gpu
def test_fused_pso_argument_checks():
    from warpsymbolic_b200 import rpn_cuda_native as ours
    g, pop, consts, X, y = _fused_case(1, 4, 10, 3, 50)
    ids = g.scalar_ids()

    def call(pop_=pop, consts_=consts, X_=X, y_=y, P=20):
        B, K = consts_.shape
        ours.fused_pso(T(pop_), T(consts_), T(X_), T(y_), torch.empty((B, K), device=DEV,
                       dtype=T(X_).dtype), torch.empty(B, device=DEV, dtype=T(X_).dtype), P, 3,
                       0.5, 1.5, 1.5, -25.0, 25.0, *ids, math.pi, math.e, 1)

    with pytest.raises(RuntimeError, match="Formula length exceeds PSO_MAX_L"):
        call(pop_=np.zeros((4, 300), np.uint8))
    with pytest.raises(RuntimeError, match="Constants exceed PSO_MAX_K"):
        call(consts_=np.zeros((4, 17), np.float32))
    with pytest.raises(RuntimeError, match="Data samples exceed PSO_MAX_D"):
        call(X_=np.zeros((2, 1025), np.float32), y_=np.zeros(1025, np.float32))
    with pytest.raises(RuntimeError, match="Particles exceed PSO_MAX_PARTICLES"):
        call(P=65)
    with pytest.raises(RuntimeError, match="float32 only"):
        call(consts_=consts.astype(np.float64), X_=X.astype(np.float64), y_=y.astype(np.float64))
