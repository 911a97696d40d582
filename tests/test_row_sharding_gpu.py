"""Row sharding on one GPU: the partial sums of row shards scored one after another, combined
with the evaluator's rules, give the losses of the whole data set scored at once."""
import numpy as np
import pytest
import torch

import ws_testlib as tl

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0") if torch.cuda.is_available() else None


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_row_shards_combine_to_the_whole(dtype):
    from warpsymbolic_b200.cuda_vm import CudaRPNVM
    from warpsymbolic_b200.sharding import RowShardedEvaluator, shard_bounds
    rng = np.random.default_rng(21)
    g = tl.GPUGrammar(num_variables=4, operators=tl.C1_OPERATORS)
    pop, consts = tl.random_population(g, 3000, 32, 6, rng, valid_only=False)
    X = rng.uniform(-3, 3, size=(4, 50_001))
    y = np.sin(X[0]) + X[1] * X[2] - X[3]
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV).to(dtype)
    P = torch.from_numpy(pop).to(DEV)
    C = T(consts)
    vm = CudaRPNVM(g, DEV)
    ev = RowShardedEvaluator(vm)
    shards = 3
    total = None
    for r in range(shards):
        s, e = shard_bounds(X.shape[1], shards, r)
        sse, ninv = ev.partial(P, T(X[:, s:e]), T(y[s:e]), C)
        part = ev.pack(sse, ninv, T(y[s:e]))
        total = part if total is None else total + part
    for loss in ("mse", "rmse"):
        got = ev.combine(total, len(pop), dtype, loss).cpu().numpy()
        want = vm.eval_fitness(P, T(X), C, T(y), policy="classic", loss=loss).cpu().numpy()
        inv = 1e15 if dtype == torch.float32 else 1e100
        bad = np.abs(want) >= inv * 0.5
        assert ((np.abs(got) >= inv * 0.5) == bad).all(), loss
        rtol = 2e-6 if dtype == torch.float32 else 1e-12
        np.testing.assert_allclose(got[~bad], want[~bad], rtol=rtol, atol=0)
        assert (~bad).sum() > 1000
    # one rank (no process group): evaluate() is the whole data set
    one = ev.evaluate(P, T(X), T(y), C, loss="rmse").cpu().numpy()
    want = vm.eval_fitness(P, T(X), C, T(y), policy="classic", loss="rmse").cpu().numpy()
    fin = np.abs(want) < 1e14
    np.testing.assert_allclose(one[fin], want[fin], rtol=2e-6 if dtype == torch.float32 else 1e-12)
