"""repair_invalid_population: this library's restatement (population.PopulationOperators) against
the reference's own GPUOperators method (src/warpsymbolic/gpu/operators.py:1496-1525), run in a
subprocess with `rpn_cuda_native` resolved to the reference extension and, separately, to the
drop-in.  Same torch seed, same input population (a quarter of its rows invalid in assorted
ways): the repaired population, the constants and the number of invalid rows are identical bit
for bit; valid rows are untouched; repaired rows pass validation.  Also with the integer-constant
option and with the variable-forcing pass enabled (which advances the torch generator).

Skipped when the reference package install (baseline/_ref) or the reference extension build
(oracle/_ref) is absent.
"""
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
HELPER = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_population_run.py")
DEV = torch.device("cuda:0") if torch.cuda.is_available() else None
needs_ref = [pytest.mark.skipif(refext.path("fastmath") is None,
                                reason="reference extension not built (oracle/build_ref.sh)"),
             pytest.mark.skipif(not os.path.isdir(os.path.join(REF_PKG, "warpsymbolic")),
                                reason="reference package not installed in baseline/_ref")]
pytestmark = [pytest.mark.gpu] + needs_ref

OPTIONS = [dict(), dict(int_consts=True), dict(var_force=0.25)]


def _inputs(tmp_path, seed):
    rng = np.random.default_rng(seed)
    g = tl.GPUGrammar(num_variables=2, operators=tl.C1_OPERATORS)
    pop, _ = tl.random_population(g, 2048, 30, 10, rng, valid_only=False)
    consts = rng.uniform(-2, 2, size=(2048, 10)).astype(np.float32)
    path = str(tmp_path / ("inp%d.npz" % seed))
    np.savez(path, population=pop, constants=consts)
    return g, pop, consts, path


def _reference(native, inp, out, seed, opts):
    cmd = [sys.executable, HELPER, "--ref-package", REF_PKG, "--native", native, "--inp", inp,
           "--out", out, "--seed", str(seed)]
    if opts.get("int_consts"):
        cmd.append("--int-consts")
    if opts.get("var_force"):
        cmd += ["--var-force", str(opts["var_force"])]
    proc = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert proc.returncode == 0, proc.stderr[-3000:]
    return np.load(out)


@pytest.mark.parametrize("opt_i", range(len(OPTIONS)))
def test_repair_matches_reference_method(tmp_path, opt_i):
    from warpsymbolic_b200.population import PopulationOperators
    opts = OPTIONS[opt_i]
    seed = 11 + opt_i
    g, pop, consts, inp = _inputs(tmp_path, seed)
    ref = _reference(refext.path("fastmath"), inp, str(tmp_path / "ref.npz"), seed, opts)
    via_dropin = _reference("dropin", inp, str(tmp_path / "dropin.npz"), seed, opts)
    assert [g.id_to_token[i] for i in sorted(g.id_to_token)] == list(ref["vocab"])

    config = {"FORCE_INTEGER_CONSTANTS": bool(opts.get("int_consts")),
              "VAR_FORCE_SEED_PERCENT": float(opts.get("var_force", 0.0))}
    torch.manual_seed(seed)
    ops = PopulationOperators(g, DEV, pop.shape[1], 2, torch.float32, config)
    p, c = torch.from_numpy(pop).to(DEV), torch.from_numpy(consts).to(DEV)
    valid_before = ops.validate(p).cpu().numpy()
    p2, c2, n = ops.repair_invalid_population(p, c)
    p2, c2 = p2.cpu().numpy(), c2.cpu().numpy()

    assert n == int(ref["n_invalid"]) == int((~valid_before).sum()) > 0
    for other in (ref, via_dropin):
        assert np.array_equal(p2, other["population"])
        assert np.array_equal(c2.view(np.uint32), other["constants"].view(np.uint32))
    # valid rows untouched; repaired rows valid and with constants in range
    assert np.array_equal(p2[valid_before], pop[valid_before])
    assert np.array_equal(c2[valid_before], consts[valid_before])
    assert ops.validate(torch.from_numpy(p2).to(DEV)).all()
    fresh = c2[~valid_before]
    assert fresh.min() >= -25.0 and fresh.max() <= 25.0
    if opts.get("int_consts"):
        assert np.array_equal(fresh, np.round(fresh))


def test_repair_of_a_valid_population_changes_nothing():
    from warpsymbolic_b200.population import PopulationOperators
    rng = np.random.default_rng(3)
    g = tl.GPUGrammar(num_variables=2, operators=tl.C1_OPERATORS)
    pop, consts = tl.random_population(g, 512, 30, 4, rng, valid_only=True)
    p, c = torch.from_numpy(pop).to(DEV), torch.from_numpy(consts).to(DEV)
    ops = PopulationOperators(g, DEV, 30, 2)
    p2, c2, n = ops.repair_invalid_population(p, c)
    assert n == 0
    assert np.array_equal(p2.cpu().numpy(), pop) and np.array_equal(c2.cpu().numpy(), consts)
