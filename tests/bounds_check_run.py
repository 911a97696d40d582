"""Runs small shapes (B <= 64, D <= 300, L <= 64) through the library this process loads --
libwarpsym.so, or the build the environment variable WARPSYM_LIB names (the bounds-checked
libwarpsym_bc.so) -- and saves every output together with the library's bounds record.
Helper of tests/test_bounds_check_gpu.py, which runs it once per build and compares.

usage: bounds_check_run.py OUT.npz
"""
import math
import os
import sys

import numpy as np
import torch

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import ws_testlib as tl  # noqa: E402

from warpsymbolic_b200 import _native as N  # noqa: E402
from warpsymbolic_b200 import constfit  # noqa: E402
from warpsymbolic_b200.cuda_vm import CudaRPNVM  # noqa: E402
from warpsymbolic_b200.grammar import GPUGrammar  # noqa: E402

DEV = torch.device("cuda:0")


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def balanced_program(g, depth, L):
    """A full binary tree of 2**depth variable leaves (+ and *): Sethi-Ullman needs depth
    registers, i.e. depth - 1 spill slots, the deepest ones in the global scratch area."""
    xs = [g.token_to_id[v] for v in g.active_variables]
    ops = [g.token_to_id['+'], g.token_to_id['*']]

    def emit(d, k):
        if d == 0:
            return [xs[k % len(xs)]]
        return emit(d - 1, 2 * k) + emit(d - 1, 2 * k + 1) + [ops[d % 2]]

    row = np.zeros(L, np.uint8)
    toks = emit(depth, 0)
    row[:len(toks)] = toks
    return row


def main(out):
    rng = np.random.default_rng(5)
    res = {}
    g = GPUGrammar(num_variables=3, operators=tl.C1_OPERATORS)
    vm = CudaRPNVM(g, DEV)
    pop, consts = tl.random_population(g, 64, 64, 6, rng, valid_only=False)
    pop[0] = balanced_program(g, 5, 64)  # 63 tokens, 4 spill slots
    pop[1] = balanced_program(g, 4, 64)
    for dtype, tag in ((np.float32, "f32"), (np.float64, "f64")):
        for D in (1, 8, 20, 33, 100, 300):
            X = rng.uniform(-2, 2, size=(3, D)).astype(dtype)
            y = (np.sin(X[0]) + X[1] * X[2]).astype(dtype)
            P, Xd, cd, yd = T(pop), T(X), T(consts.astype(dtype)), T(y)
            for policy in ("classic", "fused"):
                for strict in (0, 1):
                    r = vm.eval_fitness(P, Xd, cd, yd, strict_mode=strict, policy=policy,
                                        loss="rmse")
                    res["fit_%s_%d_%s_%d" % (tag, D, policy, strict)] = r.cpu().numpy()
        # loss and gradient: K within and beyond the register accumulators
        for K in (4, 12):
            pk, ck = tl.random_population(g, 48, 64, K, rng, valid_only=False)
            X = rng.uniform(-1.5, 1.5, size=(3, 300)).astype(dtype)
            y = (np.sin(X[0]) + 0.3 * X[1] * X[2]).astype(dtype)
            loss, grad = constfit.loss_grad(T(pk), T(X), T(ck.astype(dtype)), T(y),
                                            g.scalar_ids())
            res["lg_%s_%d_loss" % (tag, K)] = loss.cpu().numpy()
            res["lg_%s_%d_grad" % (tag, K)] = grad.cpu().numpy()
        # reference-mode adjoint
        from warpsymbolic_b200 import rpn_cuda_native as rcn
        X = rng.uniform(-1.5, 1.5, size=(3, 33)).astype(dtype)
        gout = rng.standard_normal((64, 33)).astype(dtype)
        gc = torch.zeros(consts.shape, dtype=torch.float32 if dtype == np.float32 else torch.float64,
                         device=DEV)
        rcn.eval_rpn_backward(T(pop), T(X), T(consts.astype(dtype)), T(gout), gc,
                              *g.scalar_ids(), math.pi, math.e)
        res["bwd_%s" % tag] = gc.cpu().numpy()
    torch.cuda.synchronize()
    enabled, word = N.bounds_status()
    np.savez(out, bc_enabled=np.int64(enabled), bc_word=np.uint64(word),
             lib=np.array(os.path.basename(N.LIB_PATH)), **res)


if __name__ == "__main__":
    main(sys.argv[1])
