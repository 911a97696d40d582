"""Benchmark: batched RPN program evaluation with fused per-program MSE on one or more B200s.

Workload (one step = one pass of the hot path over one batch): the evaluation-only scale test
-- 1,048,576 random valid RPN programs (lengths U{3..64}, L = 64, ops + - * / sin cos exp log
sqrt neg), 5 variables, 8 constants U[-5,5] per program, X ~ U[-3,3]^{5 x 100,000} fp32,
y from a seeded depth-5 random tree; output the per-program MSE (classic-path semantics, which
is what the reference uses at this shape).  Synthetic, seeded data; no dataset is downloaded.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun, one process per GPU): every rank evaluates its own full batch (programs
are independent; no collective on the data path), so per-GPU work is fixed ("weak" scaling);
`value` is the node-evals of all ranks / max over ranks of the timed region.
`--impl reference` times the CPU restatement of the reference evaluator (the reference has no
CPU evaluator of its own) on all host cores, on a bounded program sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)
import __graft_entry__ as entry  # noqa: E402

METRIC = "program-node evals/s"
UNIT = "node-evals/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--programs", type=int, default=1_048_576)
    ap.add_argument("--rows", type=int, default=100_000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="target CPU time of the bounded CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--config", default="eval-scale",
                    choices=["eval-scale", "batched", "serving", "serving-ramp", "kernels",
                             "constopt", "c1", "opcost"],
                    help="eval-scale: the evaluation-only scale test (default); batched: 256 "
                         "uneven problems scored by one graph-replayed launch per generation; "
                         "serving: a Poisson stream of fit/evaluate requests, continuously "
                         "batched, against one request at a time; kernels: every other kernel "
                         "of the library on its own workload, timed against its roofline; "
                         "constopt: PSO then per-program L-BFGS on 65,536 programs x 16,384 "
                         "rows; c1: the reference's own estimator and engine fitting the "
                         "plain-method workload (1024x2 rows, population 1024, 20 "
                         "generations), on this library's drop-in (--impl ours) or on the "
                         "reference extension (--impl reference); serving-ramp: sustainable "
                         "request rate of both serving paths under a p99 bound; opcost: costs "
                         "inside the "
                         "fitness evaluator (schedule sweep, per-operator rows per clock)")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="kernels: fraction of the default sizes (smaller cases for profiling)")
    ap.add_argument("--requests", type=int, default=8)
    ap.add_argument("--rate", type=float, default=20.0, help="serving: arrivals per second")
    ap.add_argument("--ramp", default="20,40,80,160,320,640,1280",
                    help="serving-ramp: arrival rates (requests/s) to serve")
    ap.add_argument("--problems", type=int, default=256)
    ap.add_argument("--generations", type=int, default=50)
    ap.add_argument("--constopt-programs", type=int, default=65_536)
    ap.add_argument("--constopt-rows", type=int, default=16_384)
    return ap.parse_args()


def load_oracle():
    import importlib.util
    spec = importlib.util.spec_from_file_location("ws_oracle_py", os.path.join(REPO, "oracle", "oracle.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def workload(args, rank):
    pkg = entry.load_package()
    from warpsymbolic_b200 import synthetic
    return synthetic.eval_scale_workload(seed=args.seed + rank, n_programs=args.programs,
                                         n_rows=args.rows)


def config_dict(args, n_gpus, wl=None):
    return {"workload": "evaluation-only scale test: %d programs (len U{3..64}, L=64), 5 vars, "
                        "K=8, D=%d rows, MSE" % (args.programs, args.rows),
            "programs_per_gpu": args.programs, "rows": args.rows, "num_vars": 5, "max_len": 64,
            "constants": 8, "ops": "+ - * / sin cos exp log sqrt neg",
            "semantics": "classic evaluate_batch path (protected ops, fp32)",
            "parallelism": "program-sharded dp%d (no collective)" % n_gpus,
            "l2": "L2 flushed (256 MB write) between timed steps; per-step CUDA events"}


# ---------------------------------------------------------------------------------------
def cpu_baseline(args, wl, n_tok, oracle, tmap):
    """Times the oracle (C++ restatement, all host threads) on a bounded program sample."""
    threads = len(os.sched_getaffinity(0))
    D = wl.X.shape[1]
    n = 8
    t = 0.0
    while True:
        t0 = time.perf_counter()
        oracle.fitness(tmap, wl.population[:n], wl.X, wl.constants[:n], wl.y, policy="classic",
                       loss="mse", nthreads=threads, timed=True)
        t = time.perf_counter() - t0
        if t > args.cpu_seconds / 4 or n >= wl.population.shape[0]:
            break
        n = min(wl.population.shape[0], n * 4)
    evals = float(n_tok[:n].sum()) * D
    return {"value": evals / t, "unit": UNIT, "cores": threads, "kind": "port",
            "build": "g++ " + " ".join(oracle.NATIVE_FLAGS) + " on this host (programs split "
                     "across threads)",
            "sample": "first %d programs x %d rows of the same workload (%.1f s)" % (n, D, t)}


# FP32-pipe, MUFU and shared-memory costs per row of each operator class, for the op-mix bound
MUFU_OPS = ("sin", "cos", "exp", "log", "sqrt", "/")
PIPE_RATE = {"fp32": 128, "mufu": 16, "smem": 32}  # operations per clock per SM


def op_mix_bound(wl, sms, f_hz):
    """The evaluator's bound on this workload's operation counts if each pipe ran at its peak
    and the interpretation itself (tape decode, dispatch) were free: one FP32 lane-op per
    operator token plus 3 per row (difference, square, sum); one MUFU op per sin, cos, exp, log,
    sqrt and division (the fast-math intrinsics: one multi-function-unit instruction each); one
    4-byte shared-memory load per variable token plus one for y.  The pipes run concurrently,
    so the slowest one bounds the launch."""
    g = wl.grammar
    counts = np.bincount(wl.population.reshape(-1), minlength=256)
    op_ids = {op: g.token_to_id[op] for op in g.operators}
    var_ids = [g.token_to_id[v] for v in g.active_variables]
    n_ops = float(sum(counts[i] for i in op_ids.values()))
    n_mufu = float(sum(counts[op_ids[o]] for o in MUFU_OPS if o in op_ids))
    n_var = float(sum(counts[i] for i in var_ids))
    B = wl.population.shape[0]
    D = wl.X.shape[1]
    work = {"fp32": (n_ops + 3.0 * B) * D, "mufu": n_mufu * D, "smem": (n_var + B) * D}
    t = {k: v / (PIPE_RATE[k] * sms * f_hz) for k, v in work.items()}
    pipe = max(t, key=t.get)
    node_evals = float(wl.n_tokens().sum()) * D
    return {"pipe": pipe, "peak_node_evals_per_s": node_evals / t[pipe],
            "per_pipe_T_node_evals_per_s": {k: node_evals / v / 1e12 for k, v in t.items()},
            "per_node_eval": {k: v / node_evals for k, v in work.items()}}


def fp64_error(wl, gpu_mse, oracle, tmap, n):
    """Relative error of the FP32 GPU MSE against the FP64 oracle (correctly rounded C-library
    operators) on the first n programs; programs invalid on either side are counted apart."""
    ref = oracle.fitness(tmap, wl.population[:n], wl.X.astype(np.float64),
                         wl.constants[:n].astype(np.float64), wl.y.astype(np.float64),
                         policy="classic", loss="mse", invalid_value=1e15)
    got = np.asarray(gpu_mse[:n], dtype=np.float64)
    ok_ref, ok_got = ref < 1e14, got < 1e14
    both = ok_ref & ok_got & (ref > 0)
    rel = np.abs(got[both] - ref[both]) / ref[both]
    # the same statistic for the FP32 oracle (IEEE C-library math): FP32's own conditioning
    f32 = oracle.fitness(tmap, wl.population[:n], wl.X, wl.constants[:n], wl.y,
                         policy="classic", loss="mse", invalid_value=1e15).astype(np.float64)
    both32 = ok_ref & (f32 < 1e14) & (ref > 0)
    rel32 = np.abs(f32[both32] - ref[both32]) / ref[both32]
    ieee = {"median_rel": float(np.median(rel32)) if rel32.size else None,
            "p99_rel": float(np.percentile(rel32, 99)) if rel32.size else None,
            "max_rel": float(rel32.max()) if rel32.size else None,
            "frac_within_1e-5": float((rel32 <= 1e-5).mean()) if rel32.size else None}
    return {"programs": int(n), "valid_both": int(both.sum()), "fp32_ieee_oracle": ieee,
            "class_mismatch": int((ok_ref != ok_got).sum()),
            "median_rel": float(np.median(rel)) if rel.size else None,
            "p99_rel": float(np.percentile(rel, 99)) if rel.size else None,
            "max_rel": float(rel.max()) if rel.size else None,
            "frac_within_1e-5": float((rel <= 1e-5).mean()) if rel.size else None,
            "note": "the GPU runs the reference's fast-math FP32 intrinsics; the oracle runs "
                    "FP64 C-library math, so ill-conditioned programs amplify the difference"}


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            p = [x.strip() for x in l.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


def profile_traffic():
    """DRAM bytes per fitness-kernel launch from the committed ncu summary (if present)."""
    p = os.path.join(REPO, "profiles", "fitness_kernel_c2.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("dram_bytes_per_launch_full"), d
    return None, None


# ---------------------------------------------------------------------------------------
def run_ours(args):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    entry.load_package()
    from warpsymbolic_b200.cuda_vm import CudaRPNVM
    from warpsymbolic_b200 import _native as N

    wl = workload(args, rank)
    n_tok = wl.n_tokens()
    D = wl.X.shape[1]
    evals_per_step = float(n_tok.sum()) * D
    vm = CudaRPNVM(wl.grammar, dev)
    pop = torch.from_numpy(wl.population).to(dev)
    consts = torch.from_numpy(wl.constants).to(dev)
    X = torch.from_numpy(wl.X).to(dev)
    y = torch.from_numpy(wl.y).to(dev)
    B, L = wl.population.shape
    out = torch.empty(B, dtype=torch.float32, device=dev)
    nbytes = N.lib().ws_fitness_workspace_bytes(B, L, N.WS_F32)
    wsp = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step(phase=0):
        vm.eval_fitness(pop, X, consts, y, policy="classic", loss="mse", out=out,
                        workspace_tensor=wsp, phase=phase)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(max(args.warmup, 3)):
        step()
    barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    ev_k = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        barrier()
        wall0 = time.perf_counter()
        for i in range(args.steps):
            flush.zero_()
            ev[i][0].record(stream)
            step()
            ev[i][1].record(stream)
        barrier()
        wall = time.perf_counter() - wall0
        # the dominant kernel alone: compile once, then time evaluate-only launches
        step(phase=N.WS_PHASE_COMPILE)
        for i in range(args.steps):
            flush.zero_()
            ev_k[i][0].record(stream)
            step(phase=N.WS_PHASE_EVALUATE)
            ev_k[i][1].record(stream)
        barrier()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    kern_ms = [a.elapsed_time(b) for a, b in ev_k]
    t_total = sum(step_ms) / 1e3
    if world > 1:
        tt = torch.tensor([t_total], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_total = float(tt.item())
    total_evals = evals_per_step * args.steps * world
    value = total_evals / t_total

    # ---- end to end through the public API with host buffers -------------------------------
    e2e = None
    if not args.no_e2e:
        h_pop = torch.from_numpy(wl.population).pin_memory()
        h_c = torch.from_numpy(wl.constants).pin_memory()
        h_X = torch.from_numpy(wl.X).pin_memory()
        h_y = torch.from_numpy(wl.y).pin_memory()
        h_out = torch.empty(B, dtype=torch.float32).pin_memory()
        d_pop, d_c, d_X, d_y = (torch.empty_like(t, device=dev) for t in (h_pop, h_c, h_X, h_y))
        e_ms = []
        for i in range(args.steps + 1):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for d_, h_ in ((d_pop, h_pop), (d_c, h_c), (d_X, h_X), (d_y, h_y)):
                d_.copy_(h_, non_blocking=True)
            r = vm.eval_fitness(d_pop, d_X, d_c, d_y, policy="classic", loss="mse")
            h_out.copy_(r, non_blocking=True)
            b.record(stream)
            b.synchronize()
            if i > 0:
                e_ms.append(a.elapsed_time(b))
        h2d = sum(t.numel() * t.element_size() for t in (h_pop, h_c, h_X, h_y))
        t_e2e = sum(e_ms) / 1e3
        if world > 1:
            tt = torch.tensor([t_e2e], dtype=torch.float64, device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t_e2e = float(tt.item())
        e2e = {"value": evals_per_step * args.steps * world / t_e2e, "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(B * 4),
               "ms_per_step": 1e3 * t_e2e / args.steps}

    if rank != 0:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    # ---- roofline ---------------------------------------------------------------------------
    peaks, peak_src = measured_peaks()
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    clocks = clk.summary()
    f_max = float(peaks.get("sm_max_mhz", 1965.0))
    fp32_peak = sms * 128 * f_max * 1e6  # FP32 lane-ops/s at the max SM clock
    k_s = statistics.mean(kern_ms) / 1e3
    achieved = evals_per_step / k_s
    traffic_full, prof = profile_traffic()
    alg_bytes = B * (L + 4 * wl.constants.shape[1] + 4) + 4 * (X.shape[0] + 1) * D + 4 * B
    roof = {"bound": "fp32", "achieved": achieved / 1e12, "peak": fp32_peak / 1e12,
            "unit": "T node-evals/s (1 FP32 lane-op per node-eval)", "frac": achieved / fp32_peak,
            "traffic": traffic_full,
            "traffic_note": "ncu dram read+write of one launch on 65,536 programs, scaled x16 "
                            "to the full launch (per-program traffic)",
            "kernel": "ws::fitness_kernel<float, 16, 0> (evaluate-only launches)",
            "kernel_ms": statistics.mean(kern_ms),
            "kernel_share_of_step": statistics.mean(kern_ms) / (1e3 * t_total / args.steps),
            "peak_source": "%d SMs x 128 FP32 lanes x sm_max_mhz %.0f (%s MEASURED_PEAKS.json)"
                           % (sms, f_max, peak_src),
            "hbm": {"algorithmic_bytes_per_launch": int(alg_bytes),
                    "achieved_gbs": alg_bytes / k_s / 1e9,
                    "peak_gbs": float(peaks.get("hbm_gbs", 6650.0)),
                    "frac": alg_bytes / k_s / 1e9 / float(peaks.get("hbm_gbs", 6650.0))}}
    if clocks.get("sm_mhz"):
        roof["frac_at_sampled_clock"] = achieved / (sms * 128 * clocks["sm_mhz"] * 1e6)

    mix = op_mix_bound(wl, sms, f_max * 1e6)
    roof["op_mix"] = {"bound": mix["pipe"], "achieved": achieved / 1e12,
                      "peak": mix["peak_node_evals_per_s"] / 1e12,
                      "unit": "T node-evals/s", "frac": achieved / mix["peak_node_evals_per_s"],
                      "per_pipe_peak": mix["per_pipe_T_node_evals_per_s"],
                      "ops_per_node_eval": mix["per_node_eval"],
                      "assumes": "pipes at peak (FP32 128, MUFU 16, shared 32 four-byte loads per "
                                 "clock per SM), one MUFU op per sin/cos/exp/log/sqrt/division, "
                                 "tape decode and dispatch free"}
    cpu = None
    err64 = None
    if not args.no_cpu_baseline and world == 1:
        oracle = load_oracle()
        cpu = cpu_baseline(args, wl, n_tok, oracle, vm.token_map())
        err64 = fp64_error(wl, out.cpu().numpy(), oracle, vm.token_map(),
                           min(512, wl.population.shape[0]))

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": 1e3 * t_total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded; shapes/distributions of the evaluation-only scale test)",
            "config": config_dict(args, world),
            "node_evals_per_step_per_gpu": evals_per_step,
            "hbm_gbs": alg_bytes / (t_total / args.steps) / 1e9,
            "roofline": roof, "cpu_baseline": cpu, "fp64_error": err64, "e2e": e2e,
            "clocks": clocks,
            # per step: descriptor write, compile, sort (hist, scan, scatter), evaluator
            "gpu_launches": 6 * args.steps * world,
            "wall_s_timed_region": wall}
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(args):
    """Reference arm: the CPU restatement of the reference evaluator (all host threads)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    oracle = load_oracle()
    wl = workload(args, 0)
    n_tok = wl.n_tokens()
    entry.load_package()
    from warpsymbolic_b200 import _native as N
    from warpsymbolic_b200.grammar import PI_VAL, E_VAL
    tmap = N.TokenMap.from_args(*wl.grammar.scalar_ids(), pi_val=PI_VAL, e_val=E_VAL)
    threads = len(os.sched_getaffinity(0))
    D = wl.X.shape[1]
    # sample size: ~ cpu-seconds / (steps + warmup) per step
    per_step = max(1.0, args.cpu_seconds * 2 / max(1, args.steps + args.warmup))
    n = 4
    while True:
        t0 = time.perf_counter()
        oracle.fitness(tmap, wl.population[:n], wl.X, wl.constants[:n], wl.y, policy="classic",
                       loss="mse", nthreads=threads, timed=True)
        dt = time.perf_counter() - t0
        if dt > per_step / 3 or n >= wl.population.shape[0]:
            break
        n *= 2
    for _ in range(args.warmup):
        oracle.fitness(tmap, wl.population[:n], wl.X, wl.constants[:n], wl.y, policy="classic",
                       loss="mse", nthreads=threads, timed=True)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.fitness(tmap, wl.population[:n], wl.X, wl.constants[:n], wl.y, policy="classic",
                       loss="mse", nthreads=threads, timed=True)
        ts.append(time.perf_counter() - t0)
    evals = float(n_tok[:n].sum()) * D
    value = evals * len(ts) / sum(ts)
    sample = "first %d of %d programs x %d rows per step" % (n, wl.population.shape[0], D)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(ts) / len(ts), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": config_dict(args, world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "build": "g++ " + " ".join(oracle.NATIVE_FLAGS) + " on this host",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference has no CPU evaluator (rpn_kernels.cu:10,382 rejects CPU "
                    "tensors); this arm times the C++ restatement of its evaluator"}
    print(json.dumps(line), flush=True)


def run_batched(args):
    """Batched uneven instances: `--problems` independent problems (rows log-uniform in
    [100, 100,000], 1..10 variables, X ~ U[-4,4], targets from depth 3-6 trees with 1% relative
    noise), 2,048 programs each (lengths U{3..64}); one generation = every problem's population
    scored (MSE) by one CUDA-graph replay of the batched pipeline (tile schedule chosen by the
    autotuner).  Beside it: the plain path -- one single-problem call per problem -- on the same
    data, and the end-to-end figure with populations and constants copied from pinned host
    memory and all losses copied back every generation."""
    import torch
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    entry.load_package()
    from warpsymbolic_b200 import synthetic, batch
    from warpsymbolic_b200.cuda_vm import CudaRPNVM
    wl = synthetic.batched_workload(seed=args.seed, n_problems=args.problems)
    evals = wl.n_node_evals()
    tot = sum(p.population.shape[0] for p in wl.problems)
    L, K = wl.problems[0].population.shape[1], wl.problems[0].constants.shape[1]
    # populations and constants of all problems: views of one buffer each (one copy per step)
    h_pop = torch.from_numpy(np.concatenate([p.population for p in wl.problems])).pin_memory()
    h_c = torch.from_numpy(np.concatenate([p.constants for p in wl.problems])).pin_memory()
    d_pop, d_c = h_pop.to(dev), h_c.to(dev)
    probs, off = [], 0
    for p in wl.problems:
        B = p.population.shape[0]
        probs.append(batch.BatchProblem(d_pop[off:off + B], torch.from_numpy(p.X).to(dev),
                                        torch.from_numpy(p.y).to(dev), d_c[off:off + B], p.grammar))
        off += B
    best, tune_ms = batch.autotune(probs, loss="mse", policy="classic", reps=2, use_cache=False)
    bf = batch.BatchedFitness(probs, loss="mse", policy="classic", schedule=best)
    graph = bf.capture()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def timed(fn, n):
        ms = []
        for _ in range(n):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        return ms

    for _ in range(max(args.warmup, 3)):
        graph.replay()
    torch.cuda.synchronize()
    with ClockSampler(0) as clk:
        g_ms = timed(graph.replay, args.generations)
    value = evals * len(g_ms) / (sum(g_ms) / 1e3)

    # plain path: one single-problem launch sequence per problem
    vms = [CudaRPNVM(p.grammar, dev) for p in probs]
    outs = [torch.empty(p.population.shape[0], dtype=torch.float32, device=dev) for p in probs]

    def plain():
        for vm, p, o in zip(vms, probs, outs):
            vm.eval_fitness(p.population, p.x, p.constants, p.y, policy="classic", loss="mse",
                            out=o)
    plain()
    torch.cuda.synchronize()
    p_ms = timed(plain, 3)
    plain_value = evals * len(p_ms) / (sum(p_ms) / 1e3)
    same = all(torch.allclose(o, bf.outputs[i], rtol=1e-6, atol=0, equal_nan=True)
               for i, o in enumerate(outs))

    # the fit loop: every generation = evaluate + breed (device GP step), one graph replay
    from warpsymbolic_b200.gp import GPStep
    init = [(p.population.clone(), p.constants.clone()) for p in probs]
    gp = GPStep(probs, bf.outputs, [args.seed * 1000 + i for i in range(len(probs))])
    fit_graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream(dev)
    side.wait_stream(stream)
    with torch.cuda.stream(side):  # warm-up outside capture, then restore and rewind
        bf.evaluate(stream=side)
        gp.step(stream=side)
        for p, (ip, ic) in zip(probs, init):
            p.population.copy_(ip)
            p.constants.copy_(ic)
        gp.set_generation(0, stream=side)
    stream.wait_stream(side)
    with torch.cuda.graph(fit_graph):
        bf.evaluate()
        gp.step()
    bf.evaluate()
    torch.cuda.synchronize()
    best0 = float(np.median([float(o.min()) for o in bf.outputs]))
    f_ms = timed(fit_graph.replay, args.generations)
    bf.evaluate()
    torch.cuda.synchronize()
    best_end = float(np.median([float(o.min()) for o in bf.outputs]))
    fit_evals = sum(float((p.population != 0).sum()) * p.x.shape[1] for p in probs)

    # plain fit: one evaluation launch sequence and one GP step per problem, per generation
    gps = [GPStep([p], [o], [i]) for i, (p, o) in enumerate(zip(probs, outs))]

    def plain_fit():
        for vm, p, o, g in zip(vms, probs, outs, gps):
            vm.eval_fitness(p.population, p.x, p.constants, p.y, policy="classic", loss="mse",
                            out=o)
            g.step()
    plain_fit()
    torch.cuda.synchronize()
    pf_ms = timed(plain_fit, 3)
    for p, (ip, ic) in zip(probs, init):
        p.population.copy_(ip)
        p.constants.copy_(ic)
    bf.evaluate()
    torch.cuda.synchronize()

    # end to end: host populations/constants in, all losses out, every generation
    h_out = torch.empty(bf.flat_out.numel(), dtype=torch.float32).pin_memory()

    def e2e_step():
        d_pop.copy_(h_pop, non_blocking=True)
        d_c.copy_(h_c, non_blocking=True)
        graph.replay()
        h_out.copy_(bf.flat_out, non_blocking=True)
    e2e_step()
    e_ms = timed(e2e_step, max(3, args.generations // 5))
    peaks, peak_src = measured_peaks()
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    f_max = float(peaks.get("sm_max_mhz", 1965.0))
    fp32_peak = sms * 128 * f_max * 1e6
    rows = [p.X.shape[1] for p in wl.problems]
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1,
            "steps": args.generations, "warmup": max(args.warmup, 3),
            "ms_per_step": statistics.mean(g_ms), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded; shapes/distributions of the batched uneven instances)",
            "config": {"workload": "batched uneven instances: %d problems x %d programs (len "
                                   "U{3..64}, L=%d, K=%d), rows log-U[100,1e5] (total %d), "
                                   "vars U{1..10}, MSE; one CUDA-graph replay per generation"
                                   % (len(probs), tot // len(probs), L, K, sum(rows)),
                       "schedule": best, "autotune_ms": tune_ms, "plan": bf.info(),
                       "l2": "L2 flushed (256 MB write) before every timed generation"},
            "node_evals_per_step": evals,
            "plain_per_problem": {"value": plain_value, "ms_per_step": statistics.mean(p_ms),
                                  "launch_sequences_per_step": len(probs),
                                  "same_losses": bool(same)},
            "roofline": {"bound": "fp32", "achieved": value / 1e12, "peak": fp32_peak / 1e12,
                         "unit": "T node-evals/s (1 FP32 lane-op per node-eval)",
                         "frac": value / fp32_peak, "traffic": None},
            "e2e": {"value": evals * len(e_ms) / (sum(e_ms) / 1e3), "unit": UNIT,
                    "h2d_bytes_per_step": int(h_pop.numel() + 4 * h_c.numel()),
                    "d2h_bytes_per_step": int(4 * h_out.numel()),
                    "ms_per_step": statistics.mean(e_ms)},
            "fit": {"what": "evaluate + device GP step (tournament 3, elitism, subtree "
                            "crossover 0.7, point mutation 0.05, constant noise) per generation, "
                            "one graph replay each",
                    "generations": args.generations,
                    "ms_per_generation": statistics.mean(f_ms),
                    "node_evals_per_s": fit_evals / (statistics.mean(f_ms) / 1e3),
                    "median_best_mse_start": best0, "median_best_mse_end": best_end,
                    "plain_ms_per_generation": statistics.mean(pf_ms),
                    "plain_launch_sequences_per_generation": 2 * len(probs)},
            "clocks": clk.summary(),
            "gpu_launches": 6 * args.generations}
    print(json.dumps(line), flush=True)
    del graph, fit_graph
    gp.close()
    for g in gps:
        g.close()
    bf.close()


def run_serving(args):
    """Serving stream: `--requests` requests arriving as a Poisson process at `--rate`/s (20 by
    default), half fits
    (population 4,096, 30 generations) and half evaluations (4,096 programs), rows log-uniform in
    [1,000, 200,000], 1..8 variables, X ~ U[-3,3], targets from depth 3-6 trees with noise
    0.01 * std(y).  Served by the continuous-batching loop (requests grouped by the work of one
    generation; per step of a group one batched evaluation and one batched GP generation, cheaper
    groups stepped more often), then by the plain path (one request at a time, one launch
    sequence per evaluation and per generation) on the same stream; every request's result is
    checked to be identical on both.  Both paths first serve the stream once untimed, so that
    neither pays first-time device allocations of these sizes in its timed run."""
    import torch
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    entry.load_package()
    from warpsymbolic_b200 import synthetic
    from warpsymbolic_b200.serving import (ContinuousBatchingServer, serve_plain,
                                           latency_summary)
    reqs = synthetic.serving_stream(seed=args.seed, n_requests=args.requests, rate=args.rate)
    # warm-up: both paths serve the same stream once, untimed, so that neither pays first-time
    # device allocations of these request sizes inside its timed run (a server that has been up)
    ContinuousBatchingServer(dev).serve(reqs, realtime=False)
    serve_plain(reqs, dev, realtime=False)
    evals = 0.0
    for r in reqs:
        n_tok = float((r.population != 0).sum())
        evals += n_tok * r.X.shape[1] * ((r.generations + 1) if r.kind == "fit" else 1)
    torch.cuda.synchronize()
    srv = ContinuousBatchingServer(dev)
    with ClockSampler(0) as clk:
        batched = srv.serve(reqs, realtime=True)
    mk_b = max(r.done for r in batched) - min(r.arrival for r in batched)
    plain = serve_plain(reqs, dev, realtime=True)
    mk_p = max(r.done for r in plain) - min(r.arrival for r in plain)
    same = True
    for a, b in zip(batched, plain):
        if a.kind == "evaluate":
            same &= bool(np.array_equal(a.losses, b.losses, equal_nan=True))
        else:
            same &= a.best_loss == b.best_loss and bool(np.array_equal(a.best_program, b.best_program))
    sb, sp = latency_summary(batched, mk_b), latency_summary(plain, mk_p)
    by_kind = {k: {"batched_p50_s": float(np.median([r.latency for r in batched if r.kind == k])),
                   "plain_p50_s": float(np.median([r.latency for r in plain if r.kind == k]))}
               for k in ("fit", "evaluate") if any(r.kind == k for r in batched)}
    line = {"metric": "served-fit p50/p99 latency and throughput vs plain", "value": sb["p99_s"],
            "unit": "s (p99 latency)", "n_gpus": 1, "steps": len(reqs), "warmup": 1,
            "ms_per_step": 1e3 * mk_b / len(reqs), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Poisson stream with the serving config's distributions)",
            "config": {"workload": "serving stream: %d requests, Poisson %g/s, fit:evaluate 1:1, "
                                   "population 4096, 30 generations, rows log-U[1e3,2e5], vars "
                                   "U{1..8}" % (len(reqs), args.rate),
                       "fits": sum(r.kind == "fit" for r in reqs), "schedule": 3},
            "batched": sb, "plain": sp, "by_kind": by_kind,
            "p99_speedup": sp["p99_s"] / sb["p99_s"], "p50_speedup": sp["p50_s"] / sb["p50_s"],
            "throughput_speedup": sb["throughput_req_s"] / sp["throughput_req_s"],
            "node_evals_per_s_batched": evals / mk_b, "node_evals_per_s_plain": evals / mk_p,
            "identical_results": same, "server": srv.stats, "clocks": clk.summary(),
            "e2e": {"value": sb["p99_s"], "unit": "s (p99 latency, host arrays in and results "
                                                    "out per request)",
                    "h2d_bytes_per_step": int(np.mean([r.population.nbytes + r.constants.nbytes
                                                       + r.X.nbytes + r.y.nbytes for r in reqs])),
                    "d2h_bytes_per_step": int(np.mean([4 * r.population.shape[0] for r in reqs]))},
            "gpu_launches": int(srv.stats.get("ticks", 0)) * 8}
    print(json.dumps(line), flush=True)


def run_serving_ramp(args):
    """Sustainable request rate under a latency bound, continuous batching against the plain
    path.  The bound is the plain path's p99 latency at the configured rate (20 requests/s).
    Then, for each arrival rate of the ramp (`--ramp`, requests/s), the same seeded stream of
    `--requests` requests (serving-config distributions: fit:evaluate 1:1, population 4,096,
    30 generations, rows log-U[1e3, 2e5], 1-8 variables) is served by both paths in real time;
    every request's result must be identical on both.  A path sustains a rate when its p99
    stays within the bound; its sustainable rate is the highest such rate of the ramp."""
    import torch
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    entry.load_package()
    from warpsymbolic_b200 import synthetic
    from warpsymbolic_b200.serving import (ContinuousBatchingServer, serve_plain,
                                           latency_summary)
    n = max(args.requests, 16)
    rates = [float(r) for r in args.ramp.split(",")]

    def same(a_res, b_res):
        ok = True
        for a, b in zip(a_res, b_res):
            if a.kind == "evaluate":
                ok &= bool(np.array_equal(a.losses, b.losses, equal_nan=True))
            else:
                ok &= a.best_loss == b.best_loss and bool(np.array_equal(a.best_program,
                                                                         b.best_program))
        return ok

    def work(reqs):  # node-evals of every evaluation the stream asks for
        return sum(float((r.population != 0).sum()) * r.X.shape[1]
                   * ((r.generations + 1) if r.kind == "fit" else 1) for r in reqs)

    def serve_both(reqs):
        srv = ContinuousBatchingServer(dev)
        b = srv.serve(reqs, realtime=True)
        mk_b = max(r.done for r in b) - min(r.arrival for r in b)
        p = serve_plain(reqs, dev, realtime=True)
        mk_p = max(r.done for r in p) - min(r.arrival for r in p)
        sb, sp = latency_summary(b, mk_b), latency_summary(p, mk_p)
        w = work(reqs)
        sb["node_evals_per_s"] = w / mk_b
        sp["node_evals_per_s"] = w / mk_p
        return sb, sp, same(b, p)

    warm = synthetic.serving_stream(seed=args.seed, n_requests=n, rate=args.rate)
    ContinuousBatchingServer(dev).serve(warm, realtime=False)
    serve_plain(warm, dev, realtime=False)
    torch.cuda.synchronize()
    # the heaviest request of the stream served alone: no schedule can finish it sooner
    heavy = max(warm, key=lambda r: work([r]))
    import dataclasses
    solo = serve_plain([dataclasses.replace(heavy, arrival=0.0)], dev, realtime=False)[0]
    solo_s = solo.latency
    with ClockSampler(0) as clk:
        b0, p0, ok0 = serve_both(warm)
        bound = p0["p99_s"]
        curve = []
        identical = ok0
        for rate in rates:
            reqs = synthetic.serving_stream(seed=args.seed, n_requests=n, rate=rate)
            sb, sp, ok = serve_both(reqs)
            identical &= ok
            curve.append({"rate_req_s": rate, "batched": sb, "plain": sp, "identical": ok})
    sus = {}
    for path in ("batched", "plain"):
        good = [c["rate_req_s"] for c in curve if c[path]["p99_s"] <= bound]
        sus[path] = max(good) if good else None
    top = curve[-1]
    line = {"metric": "sustainable served request rate under a p99 bound, continuous batching "
                      "vs plain", "value": sus["batched"], "unit": "requests/s",
            "n_gpus": 1, "steps": len(rates), "warmup": 1, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Poisson streams with the serving config's distributions)",
            "config": {"workload": "serving ramp: %d requests per rate, rates %s req/s, "
                                   "fit:evaluate 1:1, population 4096, 30 generations, rows "
                                   "log-U[1e3,2e5], vars U{1..8}" % (n, args.ramp),
                       "p99_bound_s": bound,
                       "p99_bound": "plain path's p99 at %g requests/s" % args.rate},
            "heaviest_request_alone_s": solo_s,
            "heaviest_request": {"kind": heavy.kind, "rows": int(heavy.X.shape[1]),
                                 "programs": int(heavy.population.shape[0]),
                                 "generations": int(getattr(heavy, "generations", 0))},
            "sustainable_req_s": sus,
            "sustainable_ratio": (sus["batched"] / sus["plain"]
                                  if sus["batched"] and sus["plain"] else None),
            "at_configured_rate": {"batched": b0, "plain": p0},
            "at_top_rate": {"rate_req_s": top["rate_req_s"],
                            "throughput_ratio": top["batched"]["throughput_req_s"]
                            / top["plain"]["throughput_req_s"],
                            "p99_ratio": top["plain"]["p99_s"] / top["batched"]["p99_s"]},
            "curve": curve, "identical_results": identical, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def run_constopt(args):
    """Constant optimisation: 65,536 programs (lengths U{5..40}, 2..8 constants each, K = 8),
    X ~ N(0,1)^{3 x 16,384}, y from a depth-4 tree plus 1% noise.  One step = PSO (32 particles x
    20 steps; the multi-kernel path, whose evaluation is one fitness launch per step over the
    2,097,152 particle programs) followed by per-program L-BFGS (10 iterations, history 5, strong
    Wolfe, at most 20 evaluations, each one launch of loss and adjoint gradient) and the
    improvement-only acceptance, through GPUOptimizer.  Beside it: the plain path for the L-BFGS
    phase -- the reference's structure at this size (one joint torch.optim.LBFGS over
    RPNBackwardFunction: per-row evaluator writing [B, D] predictions, torch reductions, adjoint
    kernel) -- and the end-to-end figure with host arrays in and fitted constants out."""
    import torch
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    entry.load_package()
    from warpsymbolic_b200 import synthetic
    from warpsymbolic_b200.evaluation import GPUEvaluator
    from warpsymbolic_b200.optimization import GPUOptimizer
    B, D = args.constopt_programs, args.constopt_rows
    wl = synthetic.constopt_workload(seed=args.seed, n_programs=B, n_rows=D)
    n_tok = wl.n_tokens()
    tok_sum = float(n_tok.sum())
    P_, STEPS, ITERS, HIST = 32, 20, 10, 5
    ev = GPUEvaluator(wl.grammar, dev, dtype=torch.float32)
    opt = GPUOptimizer(ev, dev, dtype=torch.float32)
    h_pop = torch.from_numpy(wl.population).pin_memory()
    h_c = torch.from_numpy(wl.constants).pin_memory()
    h_X = torch.from_numpy(np.ascontiguousarray(wl.X)).pin_memory()
    h_y = torch.from_numpy(wl.y).pin_memory()
    d_pop, d_c, d_X, d_y = (t.to(dev) for t in (h_pop, h_c, h_X, h_y))
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    ev_ = lambda: torch.cuda.Event(enable_timing=True)

    def job(pop, c, X, y):
        torch.manual_seed(args.seed)
        e0, e1, e2 = ev_(), ev_(), ev_()
        e0.record(stream)
        gpos, gerr = opt.nano_pso(pop, c, X, y, steps=STEPS, num_particles=P_)
        e1.record(stream)
        new_c, errs = opt.lbfgs_optimize_top_k(pop, gpos.to(torch.float32).contiguous(), X, y,
                                               top_k=pop.shape[0], max_iter=ITERS,
                                               per_program=True, history_size=HIST)
        e2.record(stream)
        return new_c, errs, gerr, (e0, e1, e2)

    for _ in range(max(args.warmup, 1)):
        job(d_pop, d_c, d_X, d_y)
    torch.cuda.synchronize()
    before = ev.evaluate_batch(d_pop, d_X, d_y, d_c)
    pso_ms, lb_ms, evals_tot = [], [], []
    with ClockSampler(0) as clk:
        for _ in range(max(args.steps, 1)):
            flush.zero_()
            new_c, errs, gerr, (e0, e1, e2) = job(d_pop, d_c, d_X, d_y)
            e2.synchronize()
            pso_ms.append(e0.elapsed_time(e1))
            lb_ms.append(e1.elapsed_time(e2))
            evals = opt.last_lbfgs_evals.to(torch.float64).cpu().numpy()
            evals_tot.append(evals)
    pso_evals = float(STEPS) * P_ * tok_sum * D
    ev_b = evals_tot[-1]
    lbfgs_evals = float((ev_b * n_tok).sum()) * D + 2.0 * tok_sum * D  # + initial/final scoring
    step_ms = float(np.median(np.array(pso_ms) + np.array(lb_ms)))
    value = (pso_evals + lbfgs_evals) / (step_ms / 1e3)
    rounds = int(ev_b.max())
    launches = STEPS * 8 + 2 * 6 + 2 * (rounds + 1)

    # end to end: host arrays in, fitted constants and RMSE out
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    a = ev_()
    a.record(stream)
    pop_h2d, c_h2d, X_h2d, y_h2d = (t.to(dev, non_blocking=True) for t in (h_pop, h_c, h_X, h_y))
    out_c, out_e, _, _ = job(pop_h2d, c_h2d, X_h2d, y_h2d)
    res_c, res_e = out_c.cpu(), out_e.cpu()
    b = ev_()
    b.record(stream)
    b.synchronize()
    e2e_ms = a.elapsed_time(b)
    e2e_wall = time.perf_counter() - t0

    # plain path for the L-BFGS phase (joint torch L-BFGS, history 10 as the reference's fallback)
    torch.manual_seed(args.seed)
    gpos, gerr_p = opt.nano_pso(d_pop, d_c, d_X, d_y, steps=STEPS, num_particles=P_)
    gpos = gpos.to(torch.float32).contiguous()
    opt.lbfgs_optimize_top_k(d_pop[:4096], gpos[:4096], d_X, d_y, top_k=4096, max_iter=2)
    torch.cuda.synchronize()
    flush.zero_()
    pa, pb = ev_(), ev_()
    pa.record(stream)
    plain_c, plain_e = opt.lbfgs_optimize_top_k(d_pop, gpos, d_X, d_y, top_k=B, max_iter=ITERS)
    pb.record(stream)
    pb.synchronize()
    plain_ms = pa.elapsed_time(pb)

    fin = torch.isfinite(before)
    med = lambda t: float(torch.median(t[torch.isfinite(t)]).item())
    cpu = None
    if not args.no_cpu_baseline:
        oracle = load_oracle()
        tm = entry.load_package()._native.TokenMap.from_args(*wl.grammar.scalar_ids(),
                                                             pi_val=np.pi, e_val=np.e)
        n = 4
        while True:
            t0 = time.perf_counter()
            oracle.loss_grad(tm, wl.population[:n], wl.X, wl.constants[:n], wl.y)
            t = time.perf_counter() - t0
            if t > args.cpu_seconds / 4 or n >= 4096:
                break
            n *= 4
        cpu = {"value": float(n_tok[:n].sum()) * D / t, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": "loss and adjoint gradient (the L-BFGS evaluation) of the first %d "
                         "programs x %d rows, scalar C++ restatement (%.1f s)" % (n, D, t)}
    peaks, _ = measured_peaks()
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    f_max = float(peaks.get("sm_max_mhz", 1965.0))
    peak = sms * 128 * f_max * 1e6  # FP32 lane-ops/s at the max SM clock
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1,
            "steps": len(pso_ms), "warmup": max(args.warmup, 1), "ms_per_step": step_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded; the constant-optimisation config's shapes/distributions)",
            "config": {"workload": "constant optimisation: %d programs (len U{5..40}, 2..8 C), "
                                   "K=8, 3 vars, D=%d, PSO 32x20 then L-BFGS 10 it (m=5)"
                                   % (B, D),
                       "pso": "multi-kernel path, one fitness launch per step over %d particle "
                              "programs" % (B * P_),
                       "lbfgs": "per-program strong-Wolfe L-BFGS, max_eval 20, one loss+adjoint "
                                "launch per evaluation round",
                       "l2": "L2 flushed (256 MB write) before every timed step"},
            "phases_ms": {"pso": float(np.median(pso_ms)), "lbfgs": float(np.median(lb_ms))},
            "node_evals": {"pso": pso_evals, "lbfgs_forward": lbfgs_evals,
                           "note": "L-BFGS evaluations traverse each program forward and in "
                                   "reverse; counted once"},
            "pso_node_evals_per_s": pso_evals / (np.median(pso_ms) / 1e3),
            "lbfgs_node_evals_per_s": lbfgs_evals / (np.median(lb_ms) / 1e3),
            "lbfgs_evals_per_program": {"mean": float(ev_b.mean()), "max": int(ev_b.max())},
            "roofline": {"bound": "fp32-issue", "achieved": value, "peak": peak,
                         "unit": "node-evals/s", "frac": value / peak,
                         "peak_note": "1 FP32 lane-op per node-eval: %d SMs x 128 lanes x "
                                      "%.0f MHz (the max SM clock of the measured-peaks file; "
                                      "it measures no FP32 issue rate)" % (sms, f_max),
                         "traffic": None},
            "quality": {"median_rmse_initial": med(before), "median_rmse_after_pso": med(gerr),
                        "median_rmse_final": med(errs),
                        "lbfgs_improved_frac": float((errs < gerr.to(errs.dtype)).float().mean()),
                        "plain_median_rmse_final": med(plain_e),
                        "plain_lbfgs_improved_frac":
                            float((plain_e < gerr_p.to(plain_e.dtype)).float().mean())},
            "plain_lbfgs_ms": plain_ms, "lbfgs_speedup_vs_plain": plain_ms / float(np.median(lb_ms)),
            "clocks": clk.summary(),
            "e2e": {"value": (pso_evals + lbfgs_evals) / (e2e_ms / 1e3), "unit": UNIT,
                    "ms": e2e_ms, "wall_s": e2e_wall,
                    "h2d_bytes_per_step": int(h_pop.numel() + 4 * h_c.numel() + 4 * h_X.numel()
                                              + 4 * h_y.numel()),
                    "d2h_bytes_per_step": int(4 * res_c.numel() + 4 * res_e.numel())},
            "gpu_launches": launches}
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)


def run_kernels(args):
    """Every kernel beside the fitness evaluator on a workload of the benchmark configs' shapes,
    timed with CUDA events (median of 5 after 3 warm-ups, L2 flushed before each), one JSON line
    per kernel with its algorithmic bytes (HBM-bound kernels: GB/s against the measured copy
    bandwidth) or node-evals (evaluating kernels: against 1 FP32 lane-op per node-eval)."""
    import math
    import torch
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    entry.load_package()
    from warpsymbolic_b200 import synthetic, rpn_cuda_native as R
    from warpsymbolic_b200.grammar import GPUGrammar, PI_VAL, E_VAL
    from warpsymbolic_b200.simplifier import GPUSymbolicSimplifier
    from warpsymbolic_b200.batch import BatchProblem
    from warpsymbolic_b200.gp import GPStep
    peaks, _ = measured_peaks()
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    fp32 = sms * 128 * float(peaks.get("sm_max_mhz", 1965.0)) * 1e6
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    rng = np.random.default_rng(args.seed)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    sc = lambda n: max(1, int(n * args.scale))
    out = []

    def timed(name, fn, nbytes=None, evals=None, note=""):
        for _ in range(3):
            fn()
        ms = []
        for _ in range(5):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            b.synchronize()
            ms.append(a.elapsed_time(b))
        t = statistics.median(ms) / 1e3
        line = {"kernel": name, "ms": t * 1e3, "note": note}
        if nbytes is not None:
            line.update({"bound": "hbm", "algorithmic_bytes": int(nbytes),
                         "achieved_gbs": nbytes / t / 1e9, "peak_gbs": hbm,
                         "frac": nbytes / t / 1e9 / hbm})
        if evals is not None:
            line.update({"node_evals_per_s": evals / t, "fp32_lane_op_frac": evals / t / fp32})
        out.append(line)
        print(json.dumps(line), flush=True)

    g = GPUGrammar(num_variables=5, operators=synthetic.BENCH_OPERATORS)
    ids = g.scalar_ids()
    B1, L = sc(1_048_576), 64
    pop = synthetic.random_programs(g, B1, 3, 64, L, rng, max_consts=8)
    dpop = T(pop)
    ar = T(np.array(g.arities() + [0] * (256 - g.vocab_size), dtype=np.int32)[:g.vocab_size])
    valid = torch.empty(B1, dtype=torch.bool, device=dev)
    timed("validate_rpn_batch", lambda: R.validate_rpn_batch(dpop, ar, valid, 0),
          nbytes=B1 * L + B1, note="%d x %d uint8" % (B1, L))
    starts = torch.empty((B1, L), dtype=torch.int64, device=dev)
    lens = torch.empty(B1, dtype=torch.int64, device=dev)
    timed("find_subtree_ranges", lambda: R.find_subtree_ranges(dpop, ar, starts, 0, lens),
          nbytes=B1 * L * 9 + B1 * 8, note="%d x %d -> int64 starts + lengths" % (B1, L))
    pop64 = dpop.to(torch.int64)
    timed("precompute_subtree_starts", lambda: R.precompute_subtree_starts(pop64, ar, starts),
          nbytes=B1 * L * 16, note="%d x %d int64 -> int64" % (B1, L))
    fit = T(rng.uniform(0, 10, size=B1).astype(np.float32))
    ridx = T(rng.integers(0, B1, size=(B1, 4)))
    lengths = T(rng.integers(3, 64, size=B1).astype(np.float32))
    sel = torch.empty(B1, dtype=torch.int64, device=dev)
    empty = torch.empty(0, device=dev)
    timed("tournament_selection", lambda: R.tournament_selection(
        fit, empty, ridx, torch.empty(0, dtype=torch.int32, device=dev), sel, lengths),
        nbytes=B1 * (4 + 32 + 4 + 8), note="%d programs, tournament 4, parsimony lengths" % B1)
    # genetic operators
    arn = np.array(g.arities(), dtype=np.int32)
    idsv = np.arange(g.vocab_size)
    a0 = T(idsv[(arn == 0) & (idsv != 0)].astype(np.uint8))
    a1 = T(idsv[arn == 1].astype(np.uint8))
    a2 = T(idsv[arn == 2].astype(np.uint8))
    rf = T(rng.random((B1, L), dtype=np.float32))
    ri = T(rng.integers(0, 2**62, size=(B1, L)))
    mp = dpop.clone()
    timed("mutate_population", lambda: R.mutate_population(mp, rf, ri, ar, a0, a1, a2, 0.05, 0),
          nbytes=B1 * L * (1 + 4 + 8 + 1), note="%d x %d, rate 0.05" % (B1, L))
    Np = B1 // 2
    s1 = T(rng.integers(0, 30, size=Np))
    e1 = s1 + T(rng.integers(0, 20, size=Np))
    s2 = T(rng.integers(0, 30, size=Np))
    e2 = s2 + T(rng.integers(0, 20, size=Np))
    c1 = torch.empty((Np, L), dtype=torch.uint8, device=dev)
    c2 = torch.empty_like(c1)
    timed("crossover_splicing", lambda: R.crossover_splicing(dpop[:Np], dpop[Np:2 * Np], s1, e1,
                                                             s2, e2, c1, c2, 0),
          nbytes=Np * (4 * L + 32), note="%d pairs x %d" % (Np, L))
    cst = T(rng.uniform(-5, 5, size=(B1, 8)).astype(np.float32))
    timed("constant_perturbation", lambda: R.constant_perturbation(cst, 0.3, 0.1, -25.0, 25.0, 7),
          nbytes=B1 * 8 * 4 * 2, note="%d x 8 float32, rate 0.3" % B1)
    gp = torch.empty((B1, L), dtype=torch.uint8, device=dev)
    timed("generate_random_rpn", lambda: R.generate_random_rpn(gp, a0, a1, a2, 11, 0.4, 0.2, 0.4),
          nbytes=B1 * L, note="%d x %d" % (B1, L))
    brpn = torch.zeros(L, dtype=torch.uint8, device=dev)
    bc = torch.zeros(8, dtype=torch.float32, device=dev)
    br = torch.full((1,), 1e30, dtype=torch.float32, device=dev)
    bi = torch.zeros(1, dtype=torch.int32, device=dev)

    def bub():
        br.fill_(1e30)
        R.batch_update_best(dpop, cst, fit, brpn, bc, br, bi)
    timed("batch_update_best", bub, nbytes=B1 * 4, note="%d programs (one block, as the "
                                                      "reference)" % B1)
    # simplifier
    simp = GPUSymbolicSimplifier(g, dev)
    Bs = sc(262_144)
    sp = synthetic.random_programs(g, Bs, 3, 64, L, rng, max_consts=0)
    spt = T(sp)
    timed("simplify_batch", lambda: simp.simplify_batch(spt.clone(), None, max_passes=3),
          nbytes=Bs * L * 16, note="%d x %d, 3 passes (int64 round trip)" % (Bs, L))
    # constant fitting and gradients (constant-optimisation config shapes)
    g3 = GPUGrammar(num_variables=3, operators=synthetic.BENCH_OPERATORS)
    ids3 = g3.scalar_ids()
    B3, L3, K3, D3 = sc(65_536), 40, 8, 16_384
    p3 = synthetic.random_programs(g3, B3, 5, 40, L3, rng, max_consts=K3)
    X3 = T(rng.standard_normal((3, D3)).astype(np.float32))
    y3 = T(rng.standard_normal(D3).astype(np.float32))
    c3 = T(rng.uniform(-3, 3, size=(B3, K3)).astype(np.float32))
    dp3 = T(p3)
    gout = T(rng.standard_normal((B3, D3)).astype(np.float32))
    gc = torch.zeros((B3, K3), dtype=torch.float32, device=dev)
    tok3 = float((p3 != 0).sum())
    timed("eval_rpn_backward", lambda: R.eval_rpn_backward(dp3, X3, c3, gout, gc, *ids3, PI_VAL,
                                                           E_VAL),
          nbytes=4 * B3 * D3, evals=tok3 * D3,
          note="%d programs x %d rows, K=%d (bytes: grad_output)" % (B3, D3, K3))
    from warpsymbolic_b200 import constfit
    del gout
    timed("loss_grad", lambda: constfit.loss_grad(dp3, X3, c3, y3, ids3),
          evals=tok3 * D3,
          note="%d programs x %d rows, K=%d (loss and adjoint gradient, one launch + reduce)"
               % (B3, D3, K3))
    Bp, Dp = sc(8192), 1024
    Xp, yp = X3[:, :Dp].contiguous(), y3[:Dp].contiguous()
    gpos = torch.empty((Bp, K3), dtype=torch.float32, device=dev)
    gerr = torch.empty(Bp, dtype=torch.float32, device=dev)
    tokp = float((p3[:Bp] != 0).sum())
    timed("fused_pso", lambda: R.fused_pso(dp3[:Bp], c3[:Bp], Xp, yp, gpos, gerr, 32, 20, 0.7,
                                           1.5, 1.5, -25.0, 25.0, *ids3, PI_VAL, E_VAL, 3),
          evals=tokp * Dp * 32 * 21, note="%d programs, 32 particles x 20 steps, %d rows" % (Bp, Dp))
    gb = synthetic.random_programs(g3, 64, 5, 39, L3, rng, max_consts=K3,
                                   cat_weights=(0.55, 0.0, 0.45))  # the kernel's binary-only set
    gbin = T(gb)
    cl = c3[:64].clone()
    rm = torch.empty(64, dtype=torch.float32, device=dev)

    def lb():
        cl.copy_(c3[:64])
        R.lbfgs_optimize(gbin, cl, Xp, yp, rm, 10, 5, 1e-7, -25.0, 25.0, *ids3, PI_VAL, E_VAL)
    timed("lbfgs_optimize", lb, note="64 programs (the kernel's envelope), %d rows, 10 "
                                     "iterations" % Dp)
    # classic per-row interpreter (outputs every row)
    Bc, Dc = sc(4096), 100_000
    X5 = T(rng.uniform(-3, 3, size=(5, Dc)).astype(np.float32))
    cc = T(rng.uniform(-5, 5, size=(Bc, 8)).astype(np.float32))
    preds = torch.empty((Bc, Dc), dtype=torch.float32, device=dev)
    spv = torch.empty((Bc, Dc), dtype=torch.int32, device=dev)
    err = torch.empty((Bc, Dc), dtype=torch.uint8, device=dev)
    timed("eval_rpn", lambda: R.eval_rpn(dpop[:Bc], X5, cc, preds, spv, err, *ids, PI_VAL, E_VAL, 0),
          nbytes=9 * Bc * Dc, evals=float((pop[:Bc] != 0).sum()) * Dc,
          note="%d programs x %d rows (bytes: preds, sp, error outputs)" % (Bc, Dc))
    # device GP generation (batched instances config)
    wl = synthetic.batched_workload(seed=1, n_problems=sc(256), programs=2048, rows=(100, 200))
    probs = [BatchProblem(T(p.population), T(p.X), T(p.y), T(p.constants), p.grammar)
             for p in wl.problems]
    fits = [T(rng.uniform(0, 10, size=p.population.shape[0]).astype(np.float32)) for p in wl.problems]
    gps = GPStep(probs, fits, list(range(len(probs))))
    nch = sum(p.population.shape[0] for p in wl.problems)
    timed("gp_generation", gps.step, nbytes=nch * (L + 8 * 4) * 3,
          note="%d problems x 2048 children (3 launches)" % len(probs))
    gps.close()
    # diversity: hashes and variable masks, structural dedup (insert + lookup), unique count,
    # replacement positions, fitness sharing
    x0id = g.token_to_id["x0"]
    hsh = torch.empty(B1, dtype=torch.int64, device=dev)
    vpr = torch.empty(B1, dtype=torch.int32, device=dev)
    timed("compute_population_hashes", lambda: R.compute_population_hashes(dpop, hsh, vpr, 0,
                                                                           x0id, 5),
          nbytes=B1 * (L + 8 + 4), note="%d x %d" % (B1, L))
    table = torch.empty(1 << 21, dtype=torch.int64, device=dev)
    dup = torch.empty(B1, dtype=torch.int32, device=dev)
    orig = torch.empty(B1, dtype=torch.int64, device=dev)

    def dedup():
        table.fill_(-1)
        R.structural_dedup(hsh, table, dup, orig)
    timed("structural_dedup", dedup, nbytes=B1 * (8 + 4 + 8) + (1 << 21) * 8,
          note="%d hashes into a 2^21-slot table (the table reset included)" % B1)
    pos = torch.empty(B1, dtype=torch.int64, device=dev)
    nrep = torch.zeros(1, dtype=torch.int64, device=dev)
    timed("get_replacement_positions", lambda: R.get_replacement_positions(dup, pos, nrep),
          nbytes=B1 * 4, note="%d flags (one block)" % B1)
    timed("fitness_sharing_penalty", lambda: R.fitness_sharing_penalty(dpop, 4, B1 // 4, 2, 8),
          nbytes=B1 * (L + 4), note="%d programs, 4 islands" % B1)
    # evolve_generation: selection, crossover, mutation, constant operators (no PSO steps)
    Be, Le, De = sc(262_144), 40, 64
    ge = GPUGrammar(num_variables=3, operators=synthetic.BENCH_OPERATORS)
    pe = synthetic.random_programs(ge, Be, 2, Le, Le, rng, const_prob=0.4, max_consts=8)
    are = np.array(ge.arities(), dtype=np.int32)
    ide = np.arange(ge.vocab_size)
    ev = dict(pop=T(pe), c=T(rng.uniform(-2, 2, size=(Be, 8)).astype(np.float32)),
              fit=T(rng.uniform(0.1, 5.0, size=Be).astype(np.float32)),
              X=T(rng.uniform(-2, 2, size=(3, De)).astype(np.float32)),
              lens=T((pe != 0).sum(1).astype(np.float32)),
              bank=T(synthetic.random_programs(ge, 1024, 2, Le, Le, rng, max_consts=8)))
    ev["y"] = (torch.sin(ev["X"][0]) + ev["X"][1] * ev["X"][2]).contiguous()
    e64 = torch.empty(0, dtype=torch.int64, device=dev)
    ef = torch.empty(0, dtype=torch.float32, device=dev)
    argse = (T(are), T(ide[(are == 0) & (ide != 0)].astype(np.uint8)),
             T(ide[are == 1].astype(np.uint8)), T(ide[are == 2].astype(np.uint8)))
    timed("evolve_generation", lambda: R.evolve_generation(
        ev["pop"], ev["c"], ev["fit"], ef, ev["X"], ev["y"], ev["lens"], *argse, ev["bank"], ef,
        0.2, 0.5, 4, 0, 0, 0.5, 1.5, 1.5, *ge.scalar_ids(), PI_VAL, E_VAL, 4, e64, e64, e64, e64,
        12345, 3),
          nbytes=Be * (Le + 32) * 3, note="%d x %d, bank 1024, 4 islands, tournament 4, no PSO "
                                          "(selection, crossover, mutation, constants)" % (Be, Le))
    # per-program L-BFGS with adjoint gradients (loss_grad buckets + state launches)
    Bl = sc(8192)
    timed("lbfgs_adjoint", lambda: constfit.lbfgs(dp3[:Bl], X3, c3[:Bl], y3, ids3, max_iter=5,
                                                  history_size=5),
          evals=float((p3[:Bl] != 0).sum()) * D3,
          note="%d programs x %d rows, 5 iterations, history 5 (evals: one pass)" % (Bl, D3))
    print(json.dumps({"config": "kernels", "kernels": len(out)}), flush=True)


def run_plain(args):
    """The reference's WarpSymbolicRegressor.fit -> TensorGeneticEngine, unmodified, on the
    plain-method workload, with `rpn_cuda_native` resolved to this library's drop-in (--impl
    ours) or to the reference extension built from its sources (--impl reference).  A step is
    one fit of 20 generations, timed by wall clock with the device synchronised on both sides
    (the engine is host-driven: its generations interleave Python work and launches); the
    population does not shard, so N > 1 runs N independent replicas."""
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    impl = args.impl
    ref_pkg = os.path.join(REPO, "baseline", "_ref")
    metric = "plain-method generations/s (reference engine, 1024x2 rows, population 1024)"
    unit = "generations/s"
    if not os.path.isdir(os.path.join(ref_pkg, "warpsymbolic")):
        if rank == 0:
            print(json.dumps({"impl": impl, "config": "c1", "unavailable":
                              "the reference package is not installed in baseline/_ref"}))
        return
    if impl == "reference":
        import glob
        hits = glob.glob(os.path.join(REPO, "oracle", "_ref", "fastmath", "rpn_cuda_native*.so"))
        if not hits:
            if rank == 0:
                print(json.dumps({"impl": "reference", "config": "c1", "unavailable":
                                  "the reference extension is not built (oracle/build_ref.sh)"}))
            return
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    entry.load_package()
    from warpsymbolic_b200 import reference_engine as RE
    mod = RE.load_dropin() if impl == "ours" else RE.load_extension(hits[0])
    runner = RE.PlainMethodRunner(mod, ref_pkg, keep_generations=False)
    for _ in range(max(args.warmup, 3)):
        res = runner.fit()
        if res.engine_error is not None:
            raise RuntimeError("engine failed: %s" % res.engine_error)
    runner.reset_records()
    fits = []
    with ClockSampler(local) as clk:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        w0 = time.perf_counter()
        for _ in range(args.steps):
            fits.append(runner.fit())
        torch.cuda.synchronize(dev)
        wall = time.perf_counter() - w0
    if any(r.engine_error is not None or r.errors for r in fits):
        raise RuntimeError("engine failed: %s" % [(r.engine_error, r.errors) for r in fits])
    t_total = sum(r.seconds for r in fits)
    if world > 1:
        tt = torch.tensor([t_total], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_total = float(tt.item())
    gens = sum(r.generations_run for r in fits)
    value = gens * world / t_total
    per_gen = [1e3 * g for r in fits for g in r.generation_seconds]
    calls = dict(runner.rec.calls)
    n_calls = sum(calls.values())
    rows, nvars = runner.X.shape
    h2d = runner.X.size * 4 + runner.y.size * 4
    if rank == 0:
        line = {"metric": metric, "value": value, "unit": unit, "n_gpus": world,
                "steps": args.steps, "warmup": max(args.warmup, 3),
                "ms_per_step": 1e3 * t_total / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded): X ~ U[-3,3]^(1024x2), y = x0^2 + 1.5 sin(x1) + "
                        "N(0, 0.01^2)",
                "config": {"workload": "plain method: WarpSymbolicRegressor.fit, population "
                                       "1024, max 30 tokens, 20 generations, tournament 4, one "
                                       "island, no holdout, protected evaluation",
                           "step": "one fit (20 generations), wall clock, device synced",
                           "native_module": "drop-in (libwarpsym.so)" if impl == "ours"
                           else "reference extension built from its sources",
                           "parallelism": "replicas x%d" % world,
                           "l2": "inputs 12 KB (L2-resident by design of the workload)"},
                "ms_per_generation": {"median": statistics.median(per_gen),
                                      "mean": statistics.mean(per_gen),
                                      "max": max(per_gen)},
                "fit_seconds": [r.seconds for r in fits],
                "final_formula": fits[-1].formula, "best_rmse": fits[-1].best_rmse,
                "native_calls": calls,
                "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": int(h2d),
                        "d2h_bytes_per_step": None,
                        "note": "the step is already end to end: host arrays into the "
                                "estimator, the formula string out"},
                "clocks": clk.summary(), "wall_s_timed_region": wall}
        if impl == "ours":
            # every native call launches at least one of this library's kernels
            line["gpu_launches"] = n_calls
            line["gpu_launches_note"] = "drop-in calls in the timed region (a lower bound)"
        else:
            line["impl"] = "reference"
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_opcost(args):
    """Costs inside the fitness evaluator: (1) every compiled schedule on a quarter of the scale
    workload (262,144 programs x 100,000 rows), evaluate-only launches; (2) per-operator costs
    on single-operator programs (65,536 programs of 63 tokens, 100,000 rows): rows per SM clock
    for one tape instruction, against the pipe's peak."""
    import torch
    entry.load_package()
    from warpsymbolic_b200 import synthetic, _native as N
    from warpsymbolic_b200.cuda_vm import CudaRPNVM
    dev = torch.device("cuda", 0)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    peaks, _ = measured_peaks()
    f_hz = float(peaks.get("sm_max_mhz", 1965.0)) * 1e6
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    def timed(vm, pop, X, c, y, sched, reps=5):
        B, L = pop.shape
        ws = torch.empty(N.lib().ws_fitness_workspace_bytes(B, L, N.WS_F32), dtype=torch.uint8,
                         device=dev)
        out = torch.empty(B, dtype=torch.float32, device=dev)
        f = lambda ph: vm.eval_fitness(pop, X, c, y, policy="classic", loss="mse", out=out,
                                       workspace_tensor=ws, phase=ph, schedule=sched)
        f(N.WS_PHASE_COMPILE)
        for _ in range(max(args.warmup, 3)):
            f(N.WS_PHASE_EVALUATE)
        torch.cuda.synchronize()
        ms = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            f(N.WS_PHASE_EVALUATE)
            b.record()
            b.synchronize()
            ms.append(a.elapsed_time(b))
        return statistics.median(ms)

    wl = synthetic.eval_scale_workload(seed=0, n_programs=262_144, n_rows=100_000)
    vm = CudaRPNVM(wl.grammar, dev)
    evals = float(wl.n_tokens().sum()) * wl.X.shape[1]
    args_w = (T(wl.population), T(wl.X), T(wl.constants), T(wl.y))
    sched = {}
    n_row_pass = int(N.lib().ws_schedule_count()) - 5  # the last five are the small-D evaluator
    for s_ in range(n_row_pass):
        ms = timed(vm, *args_w, s_)
        sched[s_] = {"ms": ms, "T_node_evals_per_s": evals / ms / 1e9}
    g = wl.grammar
    tid = g.token_to_id
    B = 65_536
    X, y = args_w[1], args_w[3]
    cc = T(np.full((B, 8), 0.37, dtype=np.float32))

    def prog(tokens):
        p = np.zeros((B, 64), dtype=np.uint8)
        p[:, :len(tokens)] = [tid[t] for t in tokens]
        return T(p)

    cases = {}
    for u in ("sin", "cos", "exp", "log", "sqrt", "neg"):
        cases["unary " + u] = (["x0"] + [u] * 62, 62)
    for b in ("+", "-", "*", "/"):
        vec, sca = ["x0"], ["x0"]
        for i in range(31):
            vec += ["x%d" % ((i + 1) % 5), b]
            sca += ["C", b]
        cases["binary %s variable" % b] = (vec, 31)
        cases["binary %s constant" % b] = (sca, 31)
    ops = {}
    for name, (toks, n_instr) in cases.items():
        ms = timed(vm, prog(toks), X, cc, y, 0)
        ops[name] = {"ms": ms, "rows_per_sm_clock": B * 1e5 * n_instr / (ms * 1e-3 * sms * f_hz)}
    print(json.dumps({"config": "opcost", "schedules": sched, "operators": ops,
                      "pipe_peaks_rows_per_sm_clock": {"fp32 (paired f32x2: 256)": 128,
                                                       "mufu": 16}}), flush=True)


def main():
    args = parse()
    if args.config == "opcost":
        run_opcost(args)
        return
    if args.config == "c1":
        run_plain(args)
        return
    if args.config == "kernels":
        run_kernels(args)
        return
    if args.config == "serving-ramp":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "config": "serving-ramp",
                              "unavailable": "the reference has no serving loop; the plain "
                                             "one-request-at-a-time path is timed beside ours"}))
            return
        run_serving_ramp(args)
        return
    if args.config == "serving":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "config": "serving",
                              "unavailable": "the reference has no serving loop; the plain "
                                             "one-request-at-a-time path is timed beside ours"}))
            return
        run_serving(args)
        return
    if args.config == "constopt":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "config": "constopt",
                              "unavailable": "the reference's multi-kernel PSO cannot run this "
                                             "size (B*P*D > 2^31 in its evaluator); its L-BFGS "
                                             "structure is timed as the plain path beside ours"}))
            return
        run_constopt(args)
        return
    if args.config == "batched":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "config": "batched",
                              "unavailable": "the reference scores one problem per "
                                             "evaluate_batch call; no batched path to time"}))
            return
        run_batched(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
