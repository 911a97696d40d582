"""The structure oracle (oracle/ws_oracle_structure.cpp) pinned against the reference (CPU only).

Fixtures:
  golden/structure_torch.npz  outputs of the reference's torch formulations, run on CPU by
                              golden/make_structure_golden.py (validation rules, subtree-start
                              fallback, island tournament);
  golden/ref_structure.npz    outputs of the reference's CUDA kernels (its extension built from
                              source), recorded on a B200 by golden/make_ref_golden.py.
"""
import os

import numpy as np
import pytest

import ws_testlib as tl

HERE = os.path.dirname(os.path.abspath(__file__))
O = tl.oracle


def _load(name):
    p = os.path.join(HERE, "golden", name)
    if not os.path.exists(p):
        pytest.skip("fixture %s not recorded" % name)
    return np.load(p)


@pytest.mark.parametrize("case", ["v3l30", "v5l64"])
def test_validation_rules_match_reference_torch(case):
    z = _load("structure_torch.npz")
    pop, ar, ars = z[case + "_pop"], z[case + "_arity_ops"], z[case + "_arity_simp"]
    clamped = O.validate(pop, ar, 0, "clamped")
    assert np.array_equal(clamped, z[case + "_valid_clamped"])
    assert np.array_equal(clamped, z[case + "_valid_custom"])
    stack = O.validate(pop.astype(np.int64), ars, 0, "stack")
    assert np.array_equal(stack, z[case + "_valid_stack"])
    # the fixtures exercise both outcomes and the rules really differ on them
    assert 0.2 < clamped.mean() < 0.8
    assert (stack != clamped).sum() > 100


@pytest.mark.parametrize("case", ["v3l30", "v5l64"])
def test_subtree_starts_match_reference_torch_on_wellformed_rows(case):
    """The torch fallback of _get_subtree_ranges agrees with the kernel's backward scan on
    well-formed programs (on malformed ones the two reference paths differ)."""
    z = _load("structure_torch.npz")
    pop, ar = z[case + "_pop"], z[case + "_arity_ops"]
    rows = z[case + "_starts_rows"]
    starts, _ = O.subtree_ranges(pop[rows], ar, 0)
    ok = O.validate(pop[rows], ar, 0, "kernel")
    assert ok.sum() > 500
    assert np.array_equal(starts[ok], z[case + "_starts_fallback"][ok])
    # the forward recurrence of the simplifier agrees on the same rows
    pre = O.subtree_starts(pop[rows].astype(np.int64), ar)
    assert np.array_equal(pre[ok], starts[ok])


@pytest.mark.parametrize("i", [0, 1, 2])
def test_island_tournament_matches_reference_torch(i):
    z = _load("structure_torch.npz")
    fit = np.nan_to_num(z["tour%d_fitness" % i], nan=np.inf)
    assert np.array_equal(O.tournament(fit, z["tour%d_cand" % i]), z["tour%d_winner" % i])


def test_oracle_matches_reference_kernels():
    z = _load("ref_structure.npz")
    pop, ar = z["population"], z["arities"]
    assert np.array_equal(O.validate(pop, ar, 0, "kernel"), z["valid"])
    starts, lengths = O.subtree_ranges(pop, ar, 0)
    assert np.array_equal(starts, z["starts"])
    cand = O.subtree_length_candidates(pop, 0)
    assert cand[np.arange(len(pop)), z["lengths"]].all()
    gapless = np.array([not ((r[:-1] == 0) & (r[1:] != 0)).any() for r in pop])
    assert np.array_equal(lengths[gapless], z["lengths"][gapless])
    assert np.array_equal(O.subtree_starts(pop.astype(np.int64), ar), z["pre_starts"])
    fit, errs, c = z["fitness"], z["errors"], z["cand"]
    cases, lens, mad = z["cases"], z["lens"], z["mad_eps"]
    for name, kw in (("plain", {}), ("lengths", {"lengths": lens}),
                     ("cases", {"errors": errs, "cases": cases}),
                     ("cases_lengths", {"errors": errs, "cases": cases, "lengths": lens}),
                     ("cases_lengths_mad", {"errors": errs, "cases": cases, "lengths": lens,
                                            "mad_eps": mad})):
        assert np.array_equal(O.tournament(fit, c, **kw), z["sel_" + name]), name


def test_rules_on_hand_written_rows():
    """Small cases with known answers for each rule (tokens 1-2 terminals, 3 unary, 4 binary)."""
    ar = np.array([0, 0, 0, 1, 2], dtype=np.int32)
    rows = np.array([
        [1, 2, 4, 3, 0, 0],   # x y + neg         -> valid under every rule
        [1, 2, 0, 4, 0, 0],   # PAD gap           -> kernel/clamped invalid, stack valid
        [0, 1, 0, 0, 0, 0],   # leading PAD       -> token after a PAD; stack: depth 0 at 0
        [4, 1, 0, 0, 0, 0],   # underflow         -> invalid
        [1, 2, 0, 0, 0, 0],   # two results       -> invalid
        [0, 0, 0, 0, 0, 0],   # empty             -> invalid
        [9, 0, 0, 0, 0, 0],   # outside the table -> kernel: a terminal; clamped: arity[4] = 2
    ], dtype=np.uint8)
    assert O.validate(rows, ar, 0, "kernel").tolist() == [1, 0, 0, 0, 0, 0, 1]
    assert O.validate(rows, ar, 0, "clamped").tolist() == [1, 0, 0, 0, 0, 0, 0]
    assert O.validate(rows.astype(np.int64), ar, 0, "stack").tolist() == [1, 1, 0, 0, 0, 0, 0]
    starts, lengths = O.subtree_ranges(rows, ar, 0)
    assert starts[0].tolist() == [0, 1, 0, 0, -1, -1]
    assert starts[1].tolist() == [0, 1, -1, -1, -1, -1]
    assert starts[3].tolist() == [-1, 1, -1, -1, -1, -1]
    assert lengths.tolist() == [4, 2, 0, 2, 2, 0, 1]
    pre = O.subtree_starts(rows.astype(np.int64), ar)
    assert pre[0].tolist() == [0, 1, 0, 0, -1, -1]
    assert pre[1].tolist() == [0, 1, -1, 3, -1, -1]  # binary at 3: both child lengths are 0


def test_tournament_tie_rules_on_hand_written_cases():
    """Known answers for the winner rule of rpn_kernels.cu:1535-1668: a strictly lower value
    wins; within the tie epsilon (1e-9 without a case, 1e-3 with one, mad_eps[case] when given)
    the shorter program wins, but only when lengths are given; a NaN never displaces the
    incumbent, and a NaN incumbent is never displaced."""
    fit = np.array([1.0, 1.0, 0.5, 0.5, np.nan, 2.0], dtype=np.float32)
    lens = np.array([10, 5, 8, 3, 1, 1], dtype=np.float32)
    cand = np.array([[0, 1, 2, 3], [3, 2, 0, 1], [4, 5, 0, 1], [0, 4, 5, 2]], dtype=np.int64)
    assert O.tournament(fit, cand, lengths=lens).tolist() == [3, 3, 4, 2]
    assert O.tournament(fit, cand).tolist() == [2, 3, 4, 2]
    # by case: values from errors[:, case]; ties within 1e-3, or within mad_eps[case]
    errs = np.array([[1.0], [1.0004], [0.9], [0.9002], [3.0], [3.0]], dtype=np.float32)
    cases = np.zeros(2, dtype=np.int32)
    cand2 = np.array([[0, 1, 2, 3], [1, 0, 3, 2]], dtype=np.int64)
    fit2 = fit[:2]
    assert O.tournament(fit2, cand2, errors=errs, cases=cases, lengths=lens).tolist() == [3, 2]
    assert O.tournament(fit2, cand2, errors=errs, cases=cases, lengths=lens,
                        mad_eps=np.array([1e-5], dtype=np.float32)).tolist() == [2, 2]
