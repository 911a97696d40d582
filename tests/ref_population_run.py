"""Test helper, run as a subprocess: the reference's own GPUOperators.repair_invalid_population
(src/warpsymbolic/gpu/operators.py:1496-1525), imported from an installed reference package,
with `rpn_cuda_native` resolved to the module named by --native.  Reads the population and
constants from --inp (npz), seeds torch, repairs, writes population, constants and the count to
--out (npz).  One native module per process (the reference binds it at import)."""
import argparse
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import __graft_entry__ as entry  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-package", required=True)
    ap.add_argument("--native", required=True)
    ap.add_argument("--inp", required=True)
    ap.add_argument("--out", required=True)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--num-vars", type=int, default=2)
    ap.add_argument("--var-force", type=float, default=0.0)
    ap.add_argument("--int-consts", action="store_true")
    a = ap.parse_args()
    entry.load_package()
    from warpsymbolic_b200 import reference_engine as RE
    mod = RE.load_dropin() if a.native == "dropin" else RE.load_extension(a.native)
    RE.install_native(mod, a.ref_package)
    from warpsymbolic.gpu.config import GpuGlobals
    GpuGlobals.USE_OP_POW = False
    GpuGlobals.USE_OP_ABS = False
    GpuGlobals.VAR_FORCE_SEED_PERCENT = a.var_force
    GpuGlobals.FORCE_INTEGER_CONSTANTS = bool(a.int_consts)
    from warpsymbolic.gpu.grammar import GPUGrammar
    from warpsymbolic.gpu.operators import GPUOperators
    dev = torch.device("cuda:0")
    d = np.load(a.inp)
    pop = torch.from_numpy(d["population"]).to(dev)
    consts = torch.from_numpy(d["constants"]).to(dev)
    torch.manual_seed(a.seed)
    g = GPUGrammar(a.num_vars)
    ops = GPUOperators(g, dev, pop.shape[0], pop.shape[1], a.num_vars, dtype=torch.float32)
    p2, c2, n = ops.repair_invalid_population(pop, consts)
    torch.cuda.synchronize()
    np.savez(a.out, population=p2.cpu().numpy(), constants=c2.cpu().numpy(), n_invalid=int(n),
             vocab=np.array([g.id_to_token[i] for i in sorted(g.id_to_token)]))


if __name__ == "__main__":
    main()
