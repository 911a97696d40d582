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
