"""Records outputs of the REFERENCE extension (built from its sources by oracle/build_ref.sh, both
the shipped --use_fast_math build and a build without it) on seeded inputs, as golden fixtures
that pin the CPU oracle without a GPU (tests/test_oracle_pinned.py).

Runs on a machine with a GPU and oracle/_ref/ present:
    python tests/golden/make_ref_golden.py OUT_DIR
and the .npz files are then copied into tests/golden/.
"""
from __future__ import annotations

import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)
import refext  # noqa: E402
import ws_testlib as tl  # noqa: E402


def rows_case(ref, variant, strict, dev, out_dir):
    rng = np.random.default_rng(900 + strict)
    g = tl.GPUGrammar(num_variables=3, operators=tl.ALL_OPERATORS)
    pop, consts = tl.random_population(g, 400, 40, 6, rng, valid_only=False)
    X = rng.uniform(-4, 4, size=(3, 61)).astype(np.float32)
    B, D = pop.shape[0], X.shape[1]
    p = torch.empty((B, D), dtype=torch.float32, device=dev)
    s = torch.empty((B, D), dtype=torch.int32, device=dev)
    e = torch.empty((B, D), dtype=torch.uint8, device=dev)
    ref.eval_rpn(torch.from_numpy(pop).to(dev), torch.from_numpy(X).to(dev),
                 torch.from_numpy(consts).to(dev), p, s, e, *g.scalar_ids(), tl.PI_VAL, tl.E_VAL,
                 strict)
    np.savez_compressed(os.path.join(out_dir, "ref_rows_%s_s%d.npz" % (variant, strict)),
                        population=pop, X=X, constants=consts, scalar_ids=np.array(g.scalar_ids()),
                        num_variables=3, operators=np.array(tl.ALL_OPERATORS), strict=strict,
                        preds=p.cpu().numpy(), sp=s.cpu().numpy(), err=e.cpu().numpy())


def fused_case(ref, variant, dev, out_dir):
    rng = np.random.default_rng(950)
    g = tl.GPUGrammar(num_variables=2, operators=tl.C1_OPERATORS)
    pop, consts = tl.random_population(g, 1000, 30, 4, rng, valid_only=False)
    X = rng.uniform(-3, 3, size=(2, 200)).astype(np.float32)
    y = (X[0] ** 2 + 1.5 * np.sin(X[1]) + rng.normal(0, 0.01, 200)).astype(np.float32)
    out = torch.empty(1000, dtype=torch.float32, device=dev)
    ref.eval_rpn_fused(torch.from_numpy(pop).to(dev), torch.from_numpy(X).to(dev),
                       torch.from_numpy(consts).to(dev), torch.from_numpy(y).to(dev), out,
                       *g.scalar_ids(), tl.PI_VAL, tl.E_VAL, 0, 0)
    np.savez_compressed(os.path.join(out_dir, "ref_fused_%s.npz" % variant), population=pop, X=X,
                        constants=consts, y=y, scalar_ids=np.array(g.scalar_ids()),
                        num_variables=2, operators=np.array(tl.C1_OPERATORS),
                        rmse=out.cpu().numpy())


def structure_case(ref, dev, out_dir):
    """Integer kernels: validate_rpn_batch, find_subtree_ranges, precompute_subtree_starts,
    tournament_selection (identical in both builds: no floating-point arithmetic on the path
    except tournament comparisons, which are exact)."""
    from make_structure_golden import random_rows
    rng = np.random.default_rng(4242)
    g = tl.GPUGrammar(num_variables=3, operators=tl.ALL_OPERATORS)
    ar = np.zeros(g.vocab_size + 1, dtype=np.int32)
    ar[:g.vocab_size] = g.arities()
    rows = random_rows(rng, ar, 3000, 40, 0)
    pop_u8 = torch.from_numpy(rows.astype(np.uint8)).to(dev)
    ar_t = torch.from_numpy(ar).to(dev)
    valid = torch.empty(len(rows), dtype=torch.bool, device=dev)
    ref.validate_rpn_batch(pop_u8, ar_t, valid, 0)
    starts = torch.empty(rows.shape, dtype=torch.int64, device=dev)
    lengths = torch.empty(len(rows), dtype=torch.int64, device=dev)
    ref.find_subtree_ranges(pop_u8, ar_t, starts, 0, lengths)
    pre = torch.empty(rows.shape, dtype=torch.int64, device=dev)
    ref.precompute_subtree_starts(torch.from_numpy(rows).to(dev), ar_t, pre)
    B, T, n_data = 2048, 5, 37
    fit = rng.standard_normal(B).astype(np.float32) ** 2
    fit[::50] = fit[1]
    errs = np.abs(rng.standard_normal((B, n_data))).astype(np.float32)
    errs[:, 3] = np.round(errs[:, 3], 1)  # many near-ties on one case
    cand = rng.integers(0, B, size=(B, T)).astype(np.int64)
    cases = rng.integers(-1, n_data, size=B).astype(np.int32)
    lens = rng.integers(3, 40, size=B).astype(np.float32)
    mad = (rng.random(n_data) * 0.2).astype(np.float32)

    def T_(a):
        return torch.from_numpy(a).to(dev)

    e0 = torch.empty(0, dtype=torch.float32, device=dev)
    i0 = torch.empty(0, dtype=torch.int32, device=dev)
    sel = {}
    for name, (errors, rc, ln, me) in (
            ("plain", (e0, i0, e0, e0)), ("lengths", (e0, i0, T_(lens), e0)),
            ("cases", (T_(errs), T_(cases), e0, e0)),
            ("cases_lengths", (T_(errs), T_(cases), T_(lens), e0)),
            ("cases_lengths_mad", (T_(errs), T_(cases), T_(lens), T_(mad)))):
        out = torch.empty(B, dtype=torch.int64, device=dev)
        ref.tournament_selection(T_(fit), errors, T_(cand), rc, out, ln, me)
        sel["sel_" + name] = out.cpu().numpy()
    np.savez_compressed(os.path.join(out_dir, "ref_structure.npz"),
                        population=rows.astype(np.uint8), arities=ar, valid=valid.cpu().numpy(),
                        starts=starts.cpu().numpy(), lengths=lengths.cpu().numpy(),
                        pre_starts=pre.cpu().numpy(), fitness=fit, errors=errs, cand=cand,
                        cases=cases, lens=lens, mad_eps=mad, **sel)


def simplify_case(ref, dev, out_dir):
    """simplify_batch on literal-rich programs (rules fire often), one and three passes."""
    from test_simplify import _tables, literal_rich
    g = tl.GPUGrammar(num_variables=3, operators=tl.ALL_OPERATORS)
    pop = literal_rich(g, 3000, 48, 4343)
    ar, vt, li, lv, ids = _tables(g)
    args = [torch.from_numpy(a).to(dev) for a in (ar, vt, li, lv)]
    outs = {}
    for passes in (1, 3):
        t = torch.from_numpy(pop.copy()).to(dev)
        ref.simplify_batch(t, *args, passes, *[int(v) for v in ids])
        outs["out_p%d" % passes] = t.cpu().numpy()
    np.savez_compressed(os.path.join(out_dir, "ref_simplify.npz"), population=pop, arities=ar,
                        val_table=vt, literal_ids=li, literal_vals=lv, ids=ids, **outs)


def main():
    """One process per build variant: both builds export the same symbols, so loading them into
    one process would let the first one's kernels answer for the second."""
    out_dir = sys.argv[1] if len(sys.argv) > 1 else HERE
    os.makedirs(out_dir, exist_ok=True)
    if len(sys.argv) > 2:
        variant = sys.argv[2]
        dev = torch.device("cuda:0")
        ref = refext.load(variant)
        for strict in (0, 1):
            rows_case(ref, variant, strict, dev, out_dir)
        fused_case(ref, variant, dev, out_dir)
        if variant == "fastmath":
            structure_case(ref, dev, out_dir)
            simplify_case(ref, dev, out_dir)
        print("recorded", variant)
        return
    import subprocess
    for variant in ("fastmath", "precise"):
        if refext.path(variant) is None:
            print("missing reference build:", variant)
            continue
        subprocess.run([sys.executable, os.path.abspath(__file__), out_dir, variant], check=True)


if __name__ == "__main__":
    main()
