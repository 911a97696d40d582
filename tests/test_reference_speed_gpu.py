"""Speed against the reference's own GPU path on the same inputs (B200).

The reference evaluates the evaluation-only scale workload (5 variables, 100,000 rows) with its
classic path: rpn_eval_kernel writes [B, D] predictions / stack depths / error bytes, then torch
reductions (evaluation.py:128-198), chunked so that B*D < 2^31.  The test times that path and
ours (one eval_fitness launch) on the same 4,096-program subset, checks the results agree, and
requires ours to be faster.  The measured numbers are printed (pytest -s) and written to
$WS_REPORT_DIR/reference_speed.json when that variable names a directory.
"""
import json

import numpy as np
import pytest
import torch

import refext
import ws_testlib as tl

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(refext.path("fastmath") is None,
                                 reason="reference extension not built (oracle/build_ref.sh)")]


def _time(fn, reps=3):
    fn()
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        best = min(best, a.elapsed_time(b))
    return best


def test_scale_workload_speed_vs_reference_classic_path():
    ref = refext.load("fastmath")
    from warpsymbolic_b200 import synthetic
    from warpsymbolic_b200.cuda_vm import CudaRPNVM
    dev = torch.device("cuda:0")
    wl = synthetic.eval_scale_workload(seed=5, n_programs=4096, n_rows=100_000)
    g = wl.grammar
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    pop, X, c, y = T(wl.population), T(wl.X), T(wl.constants), T(wl.y)
    vm = CudaRPNVM(g, dev)
    out = torch.empty(len(wl.population), dtype=torch.float32, device=dev)
    ours = lambda: vm.eval_fitness(pop, X, c, y, policy="classic", loss="rmse", out=out,
                                   invalid_value=1e15)
    holder = {}

    def reference():
        holder["r"] = refext.classic_rmse(ref, g.scalar_ids(), pop, X, c, y, 0, 1e15)

    t_ours = _time(ours)
    t_ref = _time(reference, reps=2)
    tl.assert_fitness_close(out.cpu().numpy(), holder["r"].cpu().numpy(), rtol=1e-5, atol=1e-7)
    evals = float(wl.n_tokens().sum()) * wl.X.shape[1]
    res = {"programs": len(wl.population), "rows": wl.X.shape[1],
           "ours_ms": t_ours, "reference_classic_ms": t_ref,
           "ours_node_evals_per_s": evals / (t_ours / 1e3),
           "reference_node_evals_per_s": evals / (t_ref / 1e3), "speedup": t_ref / t_ours}
    print(json.dumps(res))
    tl.write_report("reference_speed.json", res)
    assert t_ours < t_ref
