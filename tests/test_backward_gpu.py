"""Adjoint kernel (ws_eval_rpn_backward) on the GPU: against the CPU oracle, against the
reference extension's eval_rpn_backward on identical inputs (bit-exact per row, within summation
rounding over rows), at the torch.autograd.Function boundary with gradcheck, and on the C3
constant-fitting shape (65,536 programs x 16,384 rows) with timing against the reference."""
import json
import math

import numpy as np
import pytest
import torch

import refext
import ws_testlib as tl

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0") if torch.cuda.is_available() else None
O = tl.oracle
needs_ref = pytest.mark.skipif(refext.path("fastmath") is None,
                               reason="reference extension not built (oracle/build_ref.sh)")
DIFF_OPS = ('+', '-', '*', '/', 'sin', 'cos', 'log', 'exp')


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def tmap(g):
    """Token map with pi / e as RPNBackwardFunction passes them (math.pi, math.e)."""
    return tl.N.TokenMap.from_args(*g.scalar_ids(), pi_val=math.pi, e_val=math.e)


def ours_backward(g, pop, X, consts, gout, ids=None):
    from warpsymbolic_b200 import rpn_cuda_native as ours
    grad = torch.zeros(consts.shape, dtype=consts.dtype, device=DEV)
    ours.eval_rpn_backward(pop, X, consts, gout, grad, *(ids or g.scalar_ids()), math.pi, math.e)
    return grad


def ref_backward(ref, g, pop, X, consts, gout):
    grad = torch.zeros(consts.shape, dtype=consts.dtype, device=DEV)
    ref.eval_rpn_backward(pop, X, consts, gout, grad, *g.scalar_ids(), math.pi, math.e)
    return grad


def mixed_case(seed, B, L, K, D, dtype, ops=tl.ALL_OPERATORS, V=3, valid_only=False,
               max_consts=None):
    rng = np.random.default_rng(seed)
    g = tl.GPUGrammar(num_variables=V, operators=ops)
    if max_consts is None:
        pop, consts = tl.random_population(g, B, L, K, rng, valid_only=valid_only)
    else:
        pop = tl.synthetic.random_programs(g, B, 1, L, L, rng, max_consts=max_consts)
        consts = rng.uniform(-2, 2, size=(B, K))
    X = rng.uniform(-3, 3, size=(V, D))
    gout = rng.standard_normal((B, D))
    return g, pop, consts.astype(dtype), X.astype(dtype), gout.astype(dtype)


def _close_ref(o, r, absg, rtol, dtype):
    """Ours against the reference: scaled by the largest of sum|terms| and both results; in FP32
    pairs whose terms overflow the float range are skipped (the reference's float atomics turn
    such sums into inf or NaN depending on the order the rows arrive in)."""
    scale = np.maximum(absg, np.maximum(np.abs(np.nan_to_num(r)), np.abs(np.nan_to_num(o))))
    skip = ~(absg < 3.0e38) if dtype == np.float32 else np.zeros(absg.shape, bool)
    return skip | _close(o, r, scale, rtol)


def _close(got, want, absg, rtol):
    """Equal (infinities included), both NaN, or within rtol * sum|terms| (the rounding bound
    of any summation order)."""
    with np.errstate(invalid="ignore"):
        return (got == want) | (np.isnan(got) & np.isnan(want)) | \
            (np.abs(got - want) <= rtol * absg + 1e-30)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_backward_matches_oracle(dtype):
    g, pop, consts, X, gout = mixed_case(3, 3000, 40, 6, 300, dtype)
    want, absg = O.backward(tmap(g), pop, X, consts, gout)
    got = ours_backward(g, T(pop), T(X), T(consts), T(gout)).cpu().numpy().astype(np.float64)
    ok = _close(got, want, absg, 1e-9 if dtype == np.float64 else 1e-4)
    # FP64: GPU and host math libraries differ in the last bit, which %, pow's negative-base
    # rounding rule and tan's poles can amplify without bound on a few rows; FP32: fast-math
    # intrinsics.  Bit-level parity is established against the reference kernel instead.
    bad = np.argwhere(~ok)[:5]
    assert ok.mean() >= (0.99 if dtype == np.float64 else 0.97), \
        [(tuple(i), got[tuple(i)], want[tuple(i)], absg[tuple(i)]) for i in bad]
    if dtype == np.float64:  # slots that take no gradient stay exactly zero
        assert np.array_equal(got[absg == 0], np.zeros((absg == 0).sum()))


@pytest.mark.parametrize("B,L,K,D,min_frac", [(1, 5, 1, 1, 1.0), (7, 64, 3, 5000, 0.999),
                                              (40, 256, 8, 2000, 0.9), (5000, 12, 2, 64, 0.999),
                                              (100, 30, 40, 100, 0.999)])
def test_backward_shapes_match_oracle_f64(B, L, K, D, min_frac):
    """256-token programs nest sin / cos / exp deeply enough that last-bit differences between
    the GPU and host math libraries grow into visible ones on some rows (sin of a large argument
    is the usual amplifier): a looser fraction there."""
    # continuous operators only (see test_backward_matches_oracle for the others)
    g, pop, consts, X, gout = mixed_case(B + L, B, L, K, D, np.float64,
                                         ops=tl.C1_OPERATORS + ('abs',))
    want, absg = O.backward(tmap(g), pop, X, consts, gout)
    got = ours_backward(g, T(pop), T(X), T(consts), T(gout)).cpu().numpy()
    ok = _close(got, want, absg, 1e-9)
    bad = np.argwhere(~ok)[:5]
    assert ok.mean() >= min_frac, [(tuple(i), got[tuple(i)], want[tuple(i)], absg[tuple(i)])
                                for i in bad]


def test_backward_accumulates_into_grad_and_handles_empty_cases():
    from warpsymbolic_b200 import rpn_cuda_native as ours
    g, pop, consts, X, gout = mixed_case(9, 500, 20, 4, 100, np.float64, valid_only=True)
    P, Xt, Ct, Gt = T(pop), T(X), T(consts), T(gout)
    once = ours_backward(g, P, Xt, Ct, Gt)
    grad = once.clone()
    ours.eval_rpn_backward(P, Xt, Ct, Gt, grad, *g.scalar_ids(), math.pi, math.e)
    torch.testing.assert_close(grad, 2 * once, rtol=1e-12, atol=0, equal_nan=True)
    # K = 0: nothing to write; D = 0 and B = 0: no work
    ours.eval_rpn_backward(P, Xt, Ct[:, :0].contiguous(), Gt, torch.zeros((500, 0), device=DEV,
                           dtype=torch.float64), *g.scalar_ids(), math.pi, math.e)
    z = torch.zeros_like(Ct)
    ours.eval_rpn_backward(P, Xt[:, :0].contiguous(), Ct, Gt[:, :0].contiguous(), z,
                           *g.scalar_ids(), math.pi, math.e)
    assert not z.any()
    with pytest.raises(RuntimeError, match="256 tokens"):
        big = torch.zeros((2, 300), dtype=torch.uint8, device=DEV)
        ours.eval_rpn_backward(big, Xt, Ct[:2].contiguous(), Gt[:2].contiguous(),
                               torch.zeros_like(Ct[:2]), *g.scalar_ids(), math.pi, math.e)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_backward_without_workspace_matches_grouped_launches(dtype):
    """ws_eval_rpn_backward (one launch sized for L) against the drop-in's ws_eval_rpn_backward_ws
    (programs grouped by tape size, a launch per group): the same per-row terms, summed by blocks
    of other shapes, so equal to rounding; with D = 1 and a slot per constant token every slot
    receives one term and the two agree bit for bit."""
    import ctypes as C
    from warpsymbolic_b200 import _native as N
    from warpsymbolic_b200._tensors import dtype_code, ptr, stream_of
    for D, exact in ((1, True), (3000, False)):
        g, pop, consts, X, gout = mixed_case(21 + D, 700, 40, 12, D, dtype)
        P, Xt, Ct, Gt = T(pop), T(X), T(consts), T(gout)
        grouped = ours_backward(g, P, Xt, Ct, Gt)
        single = torch.zeros_like(Ct)
        m = tmap(g)
        N.check(N.lib().ws_eval_rpn_backward(dtype_code(Xt.dtype), ptr(P), 700, 40, ptr(Xt), 3, D,
                                             ptr(Ct), 12, ptr(Gt), ptr(single), C.byref(m),
                                             stream_of(Xt)))
        if exact:
            assert torch.equal(single.isnan(), grouped.isnan())
            fin = ~single.isnan()
            assert torch.equal(single[fin], grouped[fin])
        else:  # bounded by the sum of the terms' magnitudes (the CPU oracle's)
            _, absg = O.backward(tmap(g), pop, X.astype(np.float64), consts.astype(np.float64),
                                 gout.astype(np.float64))
            a, b = single.cpu().numpy().astype(np.float64), grouped.cpu().numpy().astype(np.float64)
            assert np.array_equal(np.isnan(a), np.isnan(b))
            inf = np.isinf(a) | np.isinf(b)
            assert np.array_equal(a[inf], b[inf])  # overflowed sums overflow alike
            fin = np.isfinite(a) & np.isfinite(b) & np.isfinite(absg)
            tol = (1e-5 if dtype == np.float32 else 1e-12) * (absg[fin] + 1e-30)
            assert (np.abs(a[fin] - b[fin]) <= tol).all()


@needs_ref
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_reference_single_row_bit_exact(dtype):
    """D = 1 and a slot per C token: the reference's atomics then add one term per slot onto
    zero, so its output is the per-row adjoint itself, which must match bit for bit."""
    ref = refext.load("fastmath")
    g, pop, consts, X, gout = mixed_case(21, 6000, 40, 12, 1, dtype, max_consts=12)
    P, Xt, Ct, Gt = T(pop), T(X), T(consts), T(gout)
    r = ref_backward(ref, g, P, Xt, Ct, Gt).cpu().numpy()
    o = ours_backward(g, P, Xt, Ct, Gt).cpu().numpy()
    same = (r == o) | (np.isnan(r) & np.isnan(o))
    assert same.all(), (np.argwhere(~same)[:5], r[~same][:5], o[~same][:5])
    assert (r != 0).sum() > 1000


@needs_ref
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_reference_many_rows(dtype):
    """Many rows: the reference sums per-row terms with float atomics in arbitrary order, this
    library in FP64 in a fixed order; both lie within the rounding of the sum."""
    ref = refext.load("fastmath")
    g, pop, consts, X, gout = mixed_case(22, 3000, 40, 6, 777, dtype)
    P, Xt, Ct, Gt = T(pop), T(X), T(consts), T(gout)
    r = ref_backward(ref, g, P, Xt, Ct, Gt).cpu().numpy().astype(np.float64)
    o = ours_backward(g, P, Xt, Ct, Gt).cpu().numpy().astype(np.float64)
    _, absg = O.backward(tmap(g), pop, X, consts, gout)
    eps = 1e-4 if dtype == np.float32 else 1e-12
    ok = _close_ref(o, r, absg, eps, dtype)
    bad = np.argwhere(~ok)[:5]
    assert ok.all(), [(tuple(i), o[tuple(i)], r[tuple(i)], absg[tuple(i)]) for i in bad]


def _smooth_programs(n):
    """FP64 programs whose constant gradients finite differences resolve (no saturated exp,
    no near-zero divisor): selected with the oracle on the CPU."""
    rng = np.random.default_rng(31)
    g = tl.GPUGrammar(num_variables=2, operators=DIFF_OPS)
    pop = tl.synthetic.random_programs(g, 400, 3, 12, 12, rng, max_consts=3)
    K, D = 3, 40
    consts = rng.uniform(-1, 1, size=(400, K))
    X = rng.uniform(-1, 1, size=(2, D))
    tm = tmap(g)
    gout = np.ones((400, D))
    grad, absg = O.backward(tm, pop, X, consts, gout)
    keep = []
    for b in range(400):
        if not (absg[b] > 0).any() or absg[b].max() > 1e4:
            continue
        okb = True
        for k in range(K):
            f = []
            for h in (1e-4, 5e-5):
                cp, cm = consts[b:b + 1].copy(), consts[b:b + 1].copy()
                cp[0, k] += h
                cm[0, k] -= h
                pp = O.eval_rows(tm, pop[b:b + 1], X, cp)[0].sum()
                pm = O.eval_rows(tm, pop[b:b + 1], X, cm)[0].sum()
                f.append((pp - pm) / (2 * h))
            okb &= abs(f[0] - f[1]) <= 1e-6 * (abs(f[1]) + 1) and \
                abs(f[1] - grad[b, k]) <= 1e-5 * (abs(f[1]) + 1)
        if okb:
            keep.append(b)
        if len(keep) == n:
            break
    return g, pop[keep], consts[keep], X


def test_autograd_function_gradcheck():
    """RPNBackwardFunction (forward: eval_rpn, backward: the adjoint kernel) through
    torch.autograd.gradcheck: the full Jacobian d preds[b, d] / d C[b, k] by central
    differences of the forward against the backward kernel, FP64."""
    from warpsymbolic_b200.autograd import RPNBackwardFunction
    from warpsymbolic_b200.cuda_vm import CudaRPNVM
    g, pop, consts, X = _smooth_programs(12)
    assert len(pop) == 12
    vm = CudaRPNVM(g, DEV)
    P, Xt = T(pop), T(X)
    y = torch.zeros(X.shape[1], dtype=torch.float64, device=DEV)
    c = T(consts).requires_grad_(True)
    assert torch.autograd.gradcheck(lambda cc: RPNBackwardFunction.apply(P, cc, Xt, y, vm), (c,),
                                    eps=1e-6, atol=1e-6, rtol=1e-5)


def test_evaluate_with_gradients_matches_oracle():
    """loss = sum_b mean_d (pred - y)^2 (optimization.py:82-88): d loss / d C equals the adjoint
    with grad_output = 2 (pred - y) / D."""
    from warpsymbolic_b200.autograd import evaluate_with_gradients
    from warpsymbolic_b200.cuda_vm import CudaRPNVM
    g, pop, consts, X, _ = mixed_case(5, 800, 30, 5, 256, np.float64, valid_only=True)
    vm = CudaRPNVM(g, DEV)
    y = np.sin(X[0]) + X[1]
    c = T(consts).requires_grad_(True)
    loss, rmse = evaluate_with_gradients(T(pop), c, T(X), T(y), vm)
    loss.backward()
    preds, sp, err = O.eval_rows(tmap(g), pop, X, consts)
    gout = 2.0 * (preds - y[None, :]) / X.shape[1]
    want, absg = O.backward(tmap(g), pop, X, consts, gout)
    got = c.grad.cpu().numpy()
    ok = _close(got, want, absg, 1e-8)
    assert ok.mean() >= 0.995
    assert torch.isfinite(rmse).any()


@needs_ref
def test_constant_fitting_shape_speed_vs_reference():
    """C3 shape: 65,536 programs of <= 40 tokens with 2-8 constants, 16,384 rows, FP32.
    Checks 256 sampled programs against the oracle and times ours against the reference's
    eval_rpn_backward (one thread per (program, row) with per-row atomics)."""
    ref = refext.load("fastmath")
    B, L, K, D = 65536, 40, 8, 16384
    rng = np.random.default_rng(64)
    g = tl.GPUGrammar(num_variables=3, operators=tl.C1_OPERATORS)
    pop = tl.synthetic.random_programs(g, B, 5, L, L, rng, max_consts=8)
    consts = rng.uniform(-3, 3, size=(B, K)).astype(np.float32)
    X = rng.standard_normal((3, D)).astype(np.float32)
    P, Xt, Ct = T(pop), T(X), T(consts)
    G = torch.randn((B, D), dtype=torch.float32, device=DEV, generator=torch.Generator(
        device=DEV).manual_seed(1))
    grad_o = torch.zeros_like(Ct)
    grad_r = torch.zeros_like(Ct)
    from warpsymbolic_b200 import rpn_cuda_native as ours

    def run(mod, out):
        out.zero_()
        mod.eval_rpn_backward(P, Xt, Ct, G, out, *g.scalar_ids(), math.pi, math.e)

    times = {}
    for name, mod, out in (("ours", ours, grad_o), ("reference", ref, grad_r)):
        run(mod, out)
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(3):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            run(mod, out)
            b.record()
            b.synchronize()
            best = min(best, a.elapsed_time(b))
        times[name] = best
    sample = rng.choice(B, size=256, replace=False)
    Gs = G[torch.from_numpy(sample).to(DEV)].cpu().numpy()
    want, absg = O.backward(tmap(g), pop[sample], X, consts[sample], Gs)
    got = grad_o.cpu().numpy()[sample].astype(np.float64)
    # FP32 fast-math intrinsics (__logf, __expf, ...) against the host library: loose
    assert _close(got, want, absg, 1e-3).mean() >= 0.9
    r = grad_r.cpu().numpy()[sample].astype(np.float64)
    # the reference's float atomics over 16,384 rows: rounding up to ~1e-3 of sum|terms|
    ok = _close_ref(got, r, absg, 1e-3, np.float32)
    assert ok.all(), [(tuple(i), got[tuple(i)], r[tuple(i)]) for i in np.argwhere(~ok)[:5]]
    n_tok = float((pop != 0).sum())
    res = {"programs": B, "rows": D, "ours_ms": times["ours"],
           "reference_ms": times["reference"], "speedup": times["reference"] / times["ours"],
           "ours_node_evals_per_s": n_tok * D / (times["ours"] / 1e3)}
    print(json.dumps(res))
    tl.write_report("backward_speed.json", res)
    assert times["ours"] < times["reference"]
