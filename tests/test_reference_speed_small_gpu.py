"""Speed of `eval_rpn_fused` on the reference's own engine workload shape: 1,048,576 programs
(lengths 3..30, 2 variables, the plain-method operator set) on small data sets, against the
reference extension's `rpn_eval_fused_kernel` in the mode its autotune picks (warp mode,
launch_mode 1, for D <= 32; block mode otherwise: rpn_kernels.cu:2562-2565,
cuda_vm.py:190-242).  Identical inputs, CUDA events, median of 5 after 2 warm-up calls; the
results must agree (1e-5, same classes) and the drop-in must be faster at every D.  The table
goes to $WS_REPORT_DIR/reference_speed_small.json when that folder exists."""
import statistics

import numpy as np
import pytest
import torch

import refext
import ws_testlib as tl

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(refext.path("fastmath") is None,
                                 reason="reference extension not built (oracle/build_ref.sh)")]
DEV = torch.device("cuda:0") if torch.cuda.is_available() else None
ROWS = [8, 16, 20, 24, 32, 64, 128, 256, 819, 1024]


def _time(fn, reps=5):
    for _ in range(2):
        fn()
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        ms.append(a.elapsed_time(b))
    return statistics.median(ms)


@pytest.fixture(scope="module")
def population():
    rng = np.random.default_rng(0)
    g = tl.GPUGrammar(num_variables=2, operators=tl.C1_OPERATORS)
    B, L = 1 << 20, 30
    pop = tl.synthetic.random_programs(g, B, 3, L, L, rng, max_consts=8)
    consts = rng.uniform(-2, 2, size=(B, 10)).astype(np.float32)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)
    return g, T(pop), T(consts), int((pop != 0).sum())


def test_small_rows_faster_than_reference(population):
    g, P, C, n_tok = population
    ref = refext.load("fastmath")
    from warpsymbolic_b200 import rpn_cuda_native as ours
    rng = np.random.default_rng(1)
    table = {}
    for D in ROWS:
        X = torch.from_numpy(rng.uniform(-3, 3, size=(2, D)).astype(np.float32)).to(DEV)
        y = (X[0] ** 2 + 1.5 * torch.sin(X[1])).contiguous()
        mode = 1 if D <= 32 else 0
        r = torch.empty(P.shape[0], dtype=torch.float32, device=DEV)
        o = torch.empty_like(r)
        args = (P, X, C, y)
        t_ref = _time(lambda: ref.eval_rpn_fused(*args, r, *g.scalar_ids(), tl.PI_VAL, tl.E_VAL,
                                                 0, mode))
        t_our = _time(lambda: ours.eval_rpn_fused(*args, o, *g.scalar_ids(), tl.PI_VAL,
                                                  tl.E_VAL, 0, mode))
        tl.assert_fitness_close(o.cpu().numpy(), r.cpu().numpy(), rtol=1e-5, atol=1e-7,
                                min_frac=1.0)
        # where the drop-in's time goes: compile + length sort, and the evaluator alone
        from warpsymbolic_b200 import _native as N
        from warpsymbolic_b200.cuda_vm import CudaRPNVM
        vm = CudaRPNVM(g, DEV)
        ws = torch.empty(N.lib().ws_fitness_workspace_bytes(P.shape[0], P.shape[1], N.WS_F32),
                         dtype=torch.uint8, device=DEV)
        ph = lambda k: vm.eval_fitness(P, X, C, y, policy="fused", loss="rmse", out=o,
                                       workspace_tensor=ws, phase=k)
        t_compile = _time(lambda: ph(N.WS_PHASE_COMPILE))
        t_eval = _time(lambda: ph(N.WS_PHASE_EVALUATE))
        table[D] = {"reference_ms": t_ref, "dropin_ms": t_our, "speedup": t_ref / t_our,
                    "reference_launch_mode": mode,
                    "dropin_compile_and_sort_ms": t_compile, "dropin_evaluate_ms": t_eval,
                    "dropin_node_evals_per_s": n_tok * D / (t_our * 1e-3)}
    tl.write_report("reference_speed_small.json", table)
    slower = {D: v for D, v in table.items() if v["dropin_ms"] > v["reference_ms"]}
    assert not slower, slower
