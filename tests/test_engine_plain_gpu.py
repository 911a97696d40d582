"""The reference's own estimator and engine, unmodified, running on this library's drop-in.

`WarpSymbolicRegressor.fit` → `TensorGeneticEngine.run` (src/warpsymbolic/api/estimator.py:
805-960, src/warpsymbolic/gpu/engine.py:1519-3419) fits the plain-method workload (1024 × 2
rows, population 1024, ≤ 30 tokens, 20 generations, tournament 4, one island, no holdout) once
with `rpn_cuda_native` resolved to the drop-in and once to the reference extension compiled from
its sources, each in a process of its own (`reference_engine.py`).  Checked:

  * the run completes 20 generations with no exception raised by any native call (the
    reference's callers would swallow one and fall back to torch);
  * the engine's native call sites were exercised: evaluation (`evaluation.py:45-125` →
    `eval_rpn_fused`), PSO (`optimization.py:143` → `fused_pso`), the generation orchestrator
    (`engine.py:3021-3031` → `evolve_generation`), the best tracker (`engine.py:2254-2272`) and
    the formula tail (`engine.py:3355-3382` → `decode_rpn`);
  * every generation's population, re-scored by the reference extension and by the drop-in,
    agrees within 1e-5 relative with identical invalid classes (protected and strict);
  * every RMSE the engine received from the drop-in's `eval_rpn_fused` matches the reference
    extension on the same arguments;
  * the engine's final `decode_rpn` call gives the same string on both modules.

Skipped when the reference package install (baseline/_ref) or the reference extension build
(oracle/_ref) is absent.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

import refext
import ws_testlib as tl

REPO = tl.REPO
REF_PKG = os.path.join(REPO, "baseline", "_ref")
HARNESS = os.path.join(REPO, "regresionsimbolica-pg_b200", "reference_engine.py")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(refext.path("fastmath") is None,
                                 reason="reference extension not built (oracle/build_ref.sh)"),
              pytest.mark.skipif(not os.path.isdir(os.path.join(REF_PKG, "warpsymbolic")),
                                 reason="reference package not installed in baseline/_ref")]
DEV = torch.device("cuda:0") if torch.cuda.is_available() else None


def _run_arm(native: str, out: str):
    proc = subprocess.run([sys.executable, HARNESS, "--ref-package", REF_PKG, "--native", native,
                           "--out", out], capture_output=True, text=True, timeout=900)
    line = [l for l in proc.stdout.splitlines() if l.startswith("REFERENCE_ENGINE_RESULT ")]
    assert proc.returncode == 0 and line, (proc.stdout[-3000:], proc.stderr[-3000:])
    rec = torch.load(out, weights_only=False)
    return json.loads(line[-1].split(" ", 1)[1]), rec


@pytest.fixture(scope="module")
def runs(tmp_path_factory):
    d = tmp_path_factory.mktemp("engine")
    ours = _run_arm("dropin", str(d / "dropin.pt"))
    ref = _run_arm(refext.path("fastmath"), str(d / "ref.pt"))
    tl.write_report("engine_plain.json", {
        "dropin": {k: v for k, v in ours[0].items()},
        "reference": {k: v for k, v in ref[0].items()},
        "generations_identical": [
            bool(torch.equal(a["population"], b["population"])
                 and torch.equal(a["constants"], b["constants"]))
            for a, b in zip(ours[1]["generations"], ref[1]["generations"])]})
    return ours, ref


def _grammar(vocab):
    g = tl.GPUGrammar(num_variables=2, operators=tl.C1_OPERATORS)
    mine = [g.id_to_token[i] for i in sorted(g.id_to_token)]
    assert mine == vocab, (mine, vocab)
    return g


def test_runs_complete_on_both_modules(runs):
    for res, _ in runs:
        assert res["engine_error"] is None
        assert res["errors"] == {}
        assert res["generations_run"] == 20
        assert res["formula"]
    (ours, _), (ref, _) = runs
    assert ours["native_file"].endswith("rpn_cuda_native.py")
    assert ref["native_file"].endswith(".so")
    calls = ours["calls"]
    assert calls.get("evolve_generation") == 20
    for name in ("eval_rpn_fused", "fused_pso", "batch_update_best", "decode_rpn",
                 "generate_random_rpn", "validate_rpn_batch", "constant_perturbation"):
        assert calls.get(name, 0) >= 1, (name, calls)
    # the same call sequence on both modules
    assert ours["calls"] == ref["calls"]


@pytest.mark.parametrize("strict", [0, 1])
def test_every_generation_rescored_identically(runs, strict):
    (res, rec), _ = runs
    g = _grammar(res["vocab"])
    ref = refext.load("fastmath")
    from warpsymbolic_b200 import rpn_cuda_native as ours
    from warpsymbolic_b200.reference_engine import PlainMethodConfig, plain_method_data
    X, y = plain_method_data(PlainMethodConfig())
    x = torch.from_numpy(np.ascontiguousarray(X.T)).to(DEV)
    yt = torch.from_numpy(y).to(DEV)
    gens = rec["generations"]
    assert len(gens) == 20
    for gen in gens:
        pop = gen["population"].to(DEV).contiguous()
        consts = gen["constants"].to(DEV).float().contiguous()
        r = torch.empty(pop.shape[0], dtype=torch.float32, device=DEV)
        o = torch.empty_like(r)
        ref.eval_rpn_fused(pop, x, consts, yt, r, *g.scalar_ids(), tl.PI_VAL, tl.E_VAL, strict, 0)
        ours.eval_rpn_fused(pop, x, consts, yt, o, *g.scalar_ids(), tl.PI_VAL, tl.E_VAL, strict, 0)
        tl.assert_fitness_close(o.cpu().numpy(), r.cpu().numpy(), rtol=1e-5, atol=1e-7,
                                min_frac=1.0)


def test_engine_evaluations_match_reference(runs):
    """Each RMSE the engine received from the drop-in's `eval_rpn_fused` (through the
    reference's `GPUEvaluator.evaluate_batch` and `CudaRPNVM`), against the reference extension
    called with the same arguments."""
    (res, rec), _ = runs
    ref = refext.load("fastmath")
    evals = rec["evaluations"]
    assert len(evals) == res["calls"]["eval_rpn_fused"] >= 20
    for ev in evals:
        args = [a.to(DEV) if isinstance(a, torch.Tensor) else a for a in ev["args"]]
        held = args[4].clone()
        args[4] = torch.empty_like(held)
        ref.eval_rpn_fused(*args, **ev["kwargs"])
        tl.assert_fitness_close(held.cpu().numpy(), args[4].cpu().numpy(), rtol=1e-5,
                                atol=1e-7, min_frac=1.0)


def test_final_formula_decodes_identically(runs):
    (res, rec), _ = runs
    ref = refext.load("fastmath")
    from warpsymbolic_b200 import rpn_cuda_native as ours
    assert len(rec["decodes"]) >= 1
    for d in rec["decodes"]:
        args = (d["population"].contiguous(), d["constants"].contiguous(), d["vocab"],
                d["arities"], d["PAD_ID"], d["precision"])
        assert list(ref.decode_rpn(*args)) == d["result"] == list(ours.decode_rpn(*args))
