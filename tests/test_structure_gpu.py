"""Structure kernels on the GPU (validation, subtree starts, tournament selection), bit-exact
against the CPU oracle (oracle/ws_oracle_structure.cpp) and, when its build is present, against
the reference extension's own kernels on identical inputs.  All calls go through the C ABI (via
the drop-in module rpn_cuda_native and warpsymbolic_b200.structure)."""
import numpy as np
import pytest
import torch

import refext
import ws_testlib as tl

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0") if torch.cuda.is_available() else None
O = tl.oracle


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def populations(seed, B, L, pad_gaps=True):
    """uint8 [B, L]: well-formed programs (all operator arities), plus malformed rows."""
    rng = np.random.default_rng(seed)
    g = tl.GPUGrammar(num_variables=3, operators=tl.ALL_OPERATORS)
    if L == 0:
        return g, np.zeros((B, 0), dtype=np.uint8)
    pop, _ = tl.random_population(g, B, L, 4, rng, valid_only=(not pad_gaps) or L < 4)
    if pad_gaps and B >= 8:
        pop[::7, 0] = 0                                             # leading PAD
        pop[3::11, :] = rng.integers(0, 256, size=pop[3::11].shape)  # byte soup
    return g, pop


def arity_tables(g):
    base = np.array(g.arities() + [0], dtype=np.int32)
    odd = base.copy()
    odd[-1] = 2                      # last entry nonzero: clamped lookup differs from the kernel
    neg = base.copy()
    neg[5] = -1                      # negative arity: the literal backward scan path
    big = base.copy()
    big[6] = 1000                    # arity beyond any row length
    short = base[:8].copy()          # most tokens outside the table
    return {"grammar": base, "last_nonzero": odd, "negative": neg, "huge": big, "short": short}


SHAPES = [(3000, 30), (4096, 64), (777, 1), (129, 5), (1500, 150), (600, 256), (300, 300)]


@pytest.mark.parametrize("B,L", SHAPES)
@pytest.mark.parametrize("rule", ["kernel", "clamped", "stack"])
def test_validate_rules_bit_exact(B, L, rule):
    from warpsymbolic_b200.structure import validate_population
    g, pop = populations(10 + L, B, L)
    for tname, ar in arity_tables(g).items():
        want = O.validate(pop, ar, 0, rule)
        got = validate_population(T(pop), T(ar), 0, rule).cpu().numpy()
        assert np.array_equal(got, want), (tname, np.nonzero(got != want)[0][:10])
        got64 = validate_population(T(pop.astype(np.int64)), T(ar), 0, rule).cpu().numpy()
        assert np.array_equal(got64, want), tname


def test_validate_misaligned_rows_and_other_pad_id():
    """A population view that starts one byte into its buffer (no 4-byte row loads) and a PAD
    token other than 0."""
    from warpsymbolic_b200.structure import validate_population
    g, pop = populations(5, 2000, 64)
    ar = arity_tables(g)["grammar"]
    flat = torch.zeros(pop.size + 1, dtype=torch.uint8, device=DEV)
    view = flat[1:].view(pop.shape)
    view.copy_(T(pop))
    for pad in (0, 7):
        for rule in ("kernel", "clamped", "stack"):
            want = O.validate(pop, ar, pad, rule)
            assert np.array_equal(validate_population(view, T(ar), pad, rule).cpu().numpy(), want)


def test_validate_degenerate_shapes():
    from warpsymbolic_b200.structure import validate_population
    ar = T(np.array([0, 0, 1, 2], dtype=np.int32))
    assert validate_population(torch.zeros((0, 5), dtype=torch.uint8, device=DEV), ar).numel() == 0
    empty_rows = torch.zeros((4, 0), dtype=torch.uint8, device=DEV)
    for rule in ("kernel", "clamped", "stack"):
        assert not validate_population(empty_rows, ar, 0, rule).any()
    with pytest.raises(RuntimeError, match="non-empty"):
        validate_population(T(np.ones((2, 3), np.uint8)), T(np.zeros(0, np.int32)), 0, "clamped")


@pytest.mark.parametrize("B,L", SHAPES)
def test_subtree_ranges_bit_exact(B, L):
    from warpsymbolic_b200.structure import subtree_starts
    g, pop = populations(30 + L, B, L)
    cand = O.subtree_length_candidates(pop, 0)
    for tname, ar in arity_tables(g).items():
        want, want_len = O.subtree_ranges(pop, ar, 0)
        got, got_len = subtree_starts(T(pop), T(ar), 0, with_lengths=True)
        got, got_len = got.cpu().numpy(), got_len.cpu().numpy()
        bad = np.nonzero((got != want).any(axis=1))[0]
        assert bad.size == 0, (tname, bad[:5])
        assert np.array_equal(got_len, want_len), tname
        assert cand[np.arange(B), got_len].all()


def test_subtree_ranges_drop_in_signature():
    from warpsymbolic_b200 import rpn_cuda_native as ours
    g, pop = populations(3, 1000, 40)
    ar = T(arity_tables(g)["grammar"])
    starts = torch.empty(pop.shape, dtype=torch.int64, device=DEV)
    ours.find_subtree_ranges(T(pop), ar, starts, 0)                       # out_lengths omitted
    ours.find_subtree_ranges(T(pop), ar, starts, 0,
                             torch.empty(0, dtype=torch.long, device=DEV))  # operators.py:905
    want, _ = O.subtree_ranges(pop, arity_tables(g)["grammar"], 0)
    assert np.array_equal(starts.cpu().numpy(), want)
    with pytest.raises(RuntimeError, match="must be a CUDA tensor"):
        ours.find_subtree_ranges(torch.from_numpy(pop), ar, starts, 0)
    with pytest.raises(RuntimeError, match="expected scalar type"):
        ours.find_subtree_ranges(T(pop.astype(np.int64)), ar, starts, 0)


@pytest.mark.parametrize("B,L", SHAPES + [(200, 400)])
def test_simplifier_subtree_starts_bit_exact(B, L):
    from warpsymbolic_b200 import rpn_cuda_native as ours
    g, pop = populations(50 + L, B, L)
    pop64 = pop.astype(np.int64)
    if B > 10:
        pop64[::9, 0] = -3                                    # negative tokens
        pop64[1::13, -1] = 10_000                             # beyond the table
    for tname, ar in arity_tables(g).items():
        want = O.subtree_starts(pop64, ar)
        out = torch.empty(pop64.shape, dtype=torch.int64, device=DEV)
        ours.precompute_subtree_starts(T(pop64), T(ar), out)
        assert np.array_equal(out.cpu().numpy(), want), tname


def _tournament_inputs(seed, B, T_, n_data=29):
    rng = np.random.default_rng(seed)
    fit = (rng.standard_normal(B).astype(np.float32) ** 2)
    fit[::31] = fit[2]                                         # exact ties
    fit[5::97] = np.nan
    errs = np.abs(rng.standard_normal((B, n_data))).astype(np.float32)
    errs[:, 1] = np.round(errs[:, 1], 2)                        # near ties on one case
    cand = rng.integers(0, B, size=(B, T_)).astype(np.int64)
    cases = rng.integers(-1, n_data, size=B).astype(np.int32)
    lens = rng.integers(3, 60, size=B).astype(np.float32)
    mad = (rng.random(n_data) * 0.3).astype(np.float32)
    return fit, errs, cand, cases, lens, mad


OPTION_SETS = [(), ("lengths",), ("errors", "cases"), ("errors", "cases", "lengths"),
               ("errors", "cases", "lengths", "mad_eps"), ("cases", "lengths", "mad_eps")]


@pytest.mark.parametrize("B,T_", [(4096, 4), (1000, 1), (3333, 9)])
@pytest.mark.parametrize("opts", OPTION_SETS)
def test_tournament_bit_exact(B, T_, opts):
    from warpsymbolic_b200 import rpn_cuda_native as ours
    fit, errs, cand, cases, lens, mad = _tournament_inputs(B + T_, B, T_)
    full = {"errors": errs, "cases": cases, "lengths": lens, "mad_eps": mad}
    kw = {k: full[k] for k in opts}
    want = O.tournament(fit, cand, **kw)
    e0 = torch.empty(0, dtype=torch.float32, device=DEV)
    i0 = torch.empty(0, dtype=torch.int32, device=DEV)
    out = torch.empty(B, dtype=torch.int64, device=DEV)
    ours.tournament_selection(T(fit), T(errs) if "errors" in kw else e0, T(cand),
                              T(cases) if "cases" in kw else i0, out,
                              T(lens) if "lengths" in kw else e0,
                              T(mad) if "mad_eps" in kw else e0)
    assert np.array_equal(out.cpu().numpy(), want)


def test_tournament_tie_rules_on_hand_written_cases():
    """The tie rules' known answers (strict win, shorter on a tie only with lengths, NaN
    incumbent kept, case and MAD epsilons) through the drop-in, on the 16-byte candidate path
    (T = 4) and the scalar one (T = 3)."""
    from warpsymbolic_b200 import rpn_cuda_native as ours
    fit = np.array([1.0, 1.0, 0.5, 0.5, np.nan, 2.0], dtype=np.float32)
    lens = np.array([10, 5, 8, 3, 1, 1], dtype=np.float32)
    errs = np.array([[1.0], [1.0004], [0.9], [0.9002], [3.0], [3.0]], dtype=np.float32)
    e0 = torch.empty(0, dtype=torch.float32, device=DEV)
    i0 = torch.empty(0, dtype=torch.int32, device=DEV)

    def run(cand, errors=None, cases=None, lengths=None, mad=None):
        out = torch.empty(len(cand), dtype=torch.int64, device=DEV)
        ours.tournament_selection(T(fit[:len(cand)] if errors is not None else fit),
                                  T(errors) if errors is not None else e0, T(cand),
                                  T(cases) if cases is not None else i0, out,
                                  T(lengths) if lengths is not None else e0,
                                  T(mad) if mad is not None else e0)
        return out.cpu().tolist()

    cand = np.array([[0, 1, 2, 3], [3, 2, 0, 1], [4, 5, 0, 1], [0, 4, 5, 2]], dtype=np.int64)
    assert run(cand, lengths=lens) == [3, 3, 4, 2]
    assert run(cand) == [2, 3, 4, 2]
    assert run(np.ascontiguousarray(cand[:, 1:]), lengths=lens) == [3, 2, 1, 4]
    cand2 = np.array([[0, 1, 2, 3], [1, 0, 3, 2]], dtype=np.int64)
    cases = np.zeros(2, dtype=np.int32)
    assert run(cand2, errs, cases, lens) == [3, 2]
    assert run(cand2, errs, cases, lens, np.array([1e-5], dtype=np.float32)) == [2, 2]
    # even T on a candidate matrix whose base is not 16-byte aligned (a view one int64 into its
    # storage): the kernel's alignment check must route it to the scalar path, same winners
    buf = torch.empty(cand.size + 1, dtype=torch.int64, device=DEV)
    mis = buf[1:].view(cand.shape)
    mis.copy_(T(cand))
    assert mis.data_ptr() % 16 != 0 and mis.is_contiguous()
    out = torch.empty(len(cand), dtype=torch.int64, device=DEV)
    ours.tournament_selection(T(fit), e0, mis, i0, out, T(lens), e0)
    assert out.cpu().tolist() == [3, 3, 4, 2]


@pytest.mark.parametrize("T_", [2, 4, 8])
def test_tournament_unaligned_candidates_bit_exact(T_):
    """Random inputs with even T: the candidate matrix at a 16-byte aligned base and at a base
    8 bytes past it give the oracle's winners."""
    from warpsymbolic_b200 import rpn_cuda_native as ours
    B = 5000
    fit, errs, cand, cases, lens, mad = _tournament_inputs(B + T_, B, T_)
    want = O.tournament(fit, cand, lengths=lens)
    e0 = torch.empty(0, dtype=torch.float32, device=DEV)
    i0 = torch.empty(0, dtype=torch.int32, device=DEV)
    for shift in (0, 1):
        buf = torch.empty(cand.size + 2, dtype=torch.int64, device=DEV)
        c_t = buf[shift:shift + cand.size].view(cand.shape)
        c_t.copy_(T(cand))
        assert (c_t.data_ptr() % 16 == 0) == (shift == 0)
        out = torch.empty(B, dtype=torch.int64, device=DEV)
        ours.tournament_selection(T(fit), e0, c_t, i0, out, T(lens), e0)
        assert np.array_equal(out.cpu().numpy(), want), shift


@pytest.mark.parametrize("island_size,n_islands", [(512, 8), (100, 41), (1, 4096), (0, 3),
                                                   (4096, 1), (700, 6)])
def test_island_offset_tournament_bit_exact(island_size, n_islands):
    from warpsymbolic_b200.structure import tournament_select
    B, T_ = 4096, 5
    fit, errs, _, cases, lens, mad = _tournament_inputs(island_size, B, T_)
    rng = np.random.default_rng(n_islands)
    off = rng.integers(-(1 << 20), 1 << 20, size=(B, T_)).astype(np.int32)
    for kw in ({}, {"lengths": lens}, {"errors": errs, "cases": cases, "lengths": lens,
                                        "mad_eps": mad}):
        want = O.tournament(fit, off, island_size=island_size, n_islands=n_islands, **kw)
        got = tournament_select(T(fit), T(off), island_size=island_size, n_islands=n_islands,
                                **{k: T(v) for k, v in kw.items()})
        assert np.array_equal(got.cpu().numpy(), want), list(kw)


def test_engine_island_tournament_mirror():
    """tournament_selection_island (engine.py:899-966): winners are the first minimum of each
    slot's candidates, NaN fitness never wins against a number."""
    from warpsymbolic_b200.structure import tournament_selection_island
    fit = torch.rand(4096, device=DEV)
    fit[::3] = float("nan")
    gen = torch.Generator(device=DEV)
    gen.manual_seed(7)
    win = tournament_selection_island(fit, 8, 4, generator=gen)
    gen.manual_seed(7)
    local = torch.randint(0, 512, (8, 512, 4), device=DEV, generator=gen)
    cand = (local + torch.arange(0, 4096, 512, device=DEV).view(8, 1, 1)).view(4096, 4)
    f = torch.nan_to_num(fit, nan=float("inf"))
    want = cand.gather(1, f[cand].argmin(dim=1, keepdim=True)).squeeze(1)
    assert torch.equal(win, want)
    assert ((win // 512) == torch.arange(4096, device=DEV) // 512).all()


def test_full_size_population_properties():
    """1,048,576 programs of up to 64 tokens: a sampled slice is bit-exact against the oracle;
    on every valid row the root's subtree starts at 0, terminals start at themselves, the two
    subtree-start algorithms agree, and lengths equal the programs' token counts."""
    from warpsymbolic_b200.structure import (simplifier_subtree_starts, subtree_starts,
                                             validate_population)
    B = 1 << 20
    g = tl.GPUGrammar(num_variables=5, operators=tl.C1_OPERATORS)
    rng = np.random.default_rng(0)
    pop = tl.synthetic.random_programs(g, B, 3, 64, 64, rng, max_consts=8)
    pop[::5, 10] = 0
    ar = np.array(g.arities() + [0], dtype=np.int32)
    P, A = T(pop), T(ar)
    valid = validate_population(P, A, 0, "kernel")
    starts, lengths = subtree_starts(P, A, 0, with_lengths=True)
    pre = simplifier_subtree_starts(P, A)
    torch.cuda.synchronize()
    v = valid.cpu().numpy()
    n_tok = (pop != 0).sum(axis=1)
    assert 0.5 < v.mean() < 0.95
    s, ln, pr = starts.cpu().numpy(), lengths.cpu().numpy(), pre.cpu().numpy()
    rows = np.nonzero(v)[0]
    assert np.array_equal(ln[rows], n_tok[rows])
    assert (s[rows, ln[rows] - 1] == 0).all()
    assert np.array_equal(s[rows], pr[rows])
    term = (ar[pop] == 0) & (pop != 0)
    assert (s[term] == np.nonzero(term)[1]).all()
    sample = rng.choice(B, size=20000, replace=False)
    want, want_len = O.subtree_ranges(pop[sample], ar, 0)
    assert np.array_equal(s[sample], want)
    assert np.array_equal(ln[sample], want_len)
    assert np.array_equal(v[sample], O.validate(pop[sample], ar, 0, "kernel"))


# ---------------------------------------------------------------------------------------------
# The reference's own kernels on identical inputs.

needs_ref = pytest.mark.skipif(refext.path("fastmath") is None,
                               reason="reference extension not built (oracle/build_ref.sh)")


@needs_ref
@pytest.mark.parametrize("B,L", [(3000, 30), (4096, 64), (500, 200)])
def test_reference_kernels_identical(B, L):
    ref = refext.load("fastmath")
    from warpsymbolic_b200 import rpn_cuda_native as ours
    g, pop = populations(70 + L, B, L)
    cand = O.subtree_length_candidates(pop, 0)
    gapless = np.array([not ((r[:-1] == 0) & (r[1:] != 0)).any() for r in pop])
    for tname, ar in arity_tables(g).items():
        P, A = T(pop), T(ar)
        outs = []
        for mod in (ref, ours):
            valid = torch.empty(B, dtype=torch.bool, device=DEV)
            mod.validate_rpn_batch(P, A, valid, 0)
            starts = torch.empty((B, L), dtype=torch.int64, device=DEV)
            lengths = torch.empty(B, dtype=torch.int64, device=DEV)
            mod.find_subtree_ranges(P, A, starts, 0, lengths)
            pre = torch.empty((B, L), dtype=torch.int64, device=DEV)
            mod.precompute_subtree_starts(T(pop.astype(np.int64)), A, pre)
            outs.append((valid, starts, lengths, pre))
        torch.cuda.synchronize()
        (rv, rs, rl, rp), (ov, os_, ol, op) = outs
        assert torch.equal(rv, ov), tname
        assert torch.equal(rs, os_), tname
        assert torch.equal(rp, op), tname
        # lengths: identical on rows without PAD gaps; elsewhere both are racing candidates
        rl, ol = rl.cpu().numpy(), ol.cpu().numpy()
        assert np.array_equal(rl[gapless], ol[gapless]), tname
        assert cand[np.arange(B), ol].all() and cand[np.arange(B), rl].all()


@needs_ref
@pytest.mark.parametrize("opts", OPTION_SETS)
def test_reference_tournament_identical(opts):
    ref = refext.load("fastmath")
    from warpsymbolic_b200 import rpn_cuda_native as ours
    B, T_ = 8192, 6
    fit, errs, cand, cases, lens, mad = _tournament_inputs(11, B, T_)
    fit[7::50] = np.float32(1e-39)                               # subnormals: flushed alike
    e0 = torch.empty(0, dtype=torch.float32, device=DEV)
    i0 = torch.empty(0, dtype=torch.int32, device=DEV)
    outs = []
    for mod in (ref, ours):
        out = torch.empty(B, dtype=torch.int64, device=DEV)
        mod.tournament_selection(T(fit), T(errs) if "errors" in opts else e0, T(cand),
                                 T(cases) if "cases" in opts else i0, out,
                                 T(lens) if "lengths" in opts else e0,
                                 T(mad) if "mad_eps" in opts else e0)
        outs.append(out)
    torch.cuda.synchronize()
    assert torch.equal(outs[0], outs[1])
