"""Runs the reference package's own estimator and engine on a chosen native module.

The reference fits through `WarpSymbolicRegressor.fit` (src/warpsymbolic/api/estimator.py:
794-960) → `TensorGeneticEngine.run` (src/warpsymbolic/gpu/engine.py:1519-3419); every module
of its `gpu` package obtains the native extension through `cuda_loader.load_rpn_cuda_native()`
(src/warpsymbolic/gpu/cuda_loader.py:12-42), which falls back to `import rpn_cuda_native` when
no extension file sits in the package.  Registering a module under that name before the
reference package is imported therefore swaps the whole native layer, unmodified callers
included: this is how a user switches the reference to this library's drop-in
(`rpn_cuda_native.py` beside this file).

`RecordingModule` forwards every attribute to the wrapped module and counts the calls (and the
exceptions, which the reference's callers often swallow: `evaluation.py:123-125`,
`optimization.py:228-232`); the generation records keep each generation's population and
constants (the inputs of `evolve_generation`, `engine.py:3021-3031`) and the fitness the engine
received with them, so that they can be re-scored afterwards by any evaluator.

The reference package is not part of this library.  It is imported from a directory given by
the caller (for instance a `pip install --target` of the reference), in a process of its own:
the module cache of `cuda_loader` and the engine's global configuration (`GpuGlobals`) make one
choice of native module per process.

Command line (one process per run):
    python reference_engine.py --ref-package DIR [--native dropin|PATH.so] [--out FILE.pt]
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import math
import os
import sys
import time
import types
from dataclasses import dataclass, field
from typing import Any, Dict, List, Optional

import numpy as np
import torch

_HERE = os.path.dirname(os.path.abspath(__file__))


# ---------------------------------------------------------------------------------------------
# the module proxy
# ---------------------------------------------------------------------------------------------

class RecordingModule(types.ModuleType):
    """Stand-in for `rpn_cuda_native` that forwards to `inner` and records the calls.

    Attribute probes (`hasattr(rpn_cuda_native, 'crossover_constants')`, operators.py:1084)
    see exactly the inner module's attributes.  `evolve_generation` calls additionally keep the
    generation's population, constants and fitness (cloned to host memory), `eval_rpn_fused`
    calls their arguments with the RMSE written into `out_rmse`, and `decode_rpn` calls their
    arguments and strings."""

    def __init__(self, inner, keep_generations: bool = True):
        super().__init__("rpn_cuda_native")
        object.__setattr__(self, "_inner", inner)
        object.__setattr__(self, "calls", {})
        object.__setattr__(self, "errors", {})
        object.__setattr__(self, "generations", [])
        object.__setattr__(self, "decodes", [])
        object.__setattr__(self, "evaluations", [])
        object.__setattr__(self, "_keep", keep_generations)
        object.__setattr__(self, "__file__", getattr(inner, "__file__", "<rpn_cuda_native>"))

    def __getattr__(self, name):
        attr = getattr(object.__getattribute__(self, "_inner"), name)
        if not callable(attr) or name.startswith("__"):
            return attr
        rec = self

        def call(*args, **kwargs):
            rec.calls[name] = rec.calls.get(name, 0) + 1
            if name == "evolve_generation" and rec._keep:
                entry = {"population": args[0].detach().cpu().clone(),
                         "constants": args[1].detach().cpu().clone(),
                         "fitness": args[2].detach().cpu().clone()}
            try:
                out = attr(*args, **kwargs)
            except Exception as exc:  # recorded, then re-raised to the reference's caller
                rec.errors.setdefault(name, []).append("%s: %s" % (type(exc).__name__, exc))
                raise
            if name == "evolve_generation" and rec._keep:
                entry["new_population"] = out[0].detach().cpu().clone()
                entry["new_constants"] = out[1].detach().cpu().clone()
                entry["new_fitness"] = out[2].detach().cpu().clone()
                rec.generations.append(entry)
            elif name == "eval_rpn_fused" and rec._keep:
                # every argument (tensors to host memory) and the RMSE the engine received
                rec.evaluations.append({
                    "args": [a.detach().cpu().clone() if isinstance(a, torch.Tensor) else a
                             for a in args],
                    "kwargs": dict(kwargs)})
            elif name == "decode_rpn":
                rec.decodes.append({"population": args[0].detach().cpu().clone(),
                                    "constants": args[1].detach().cpu().clone(),
                                    "vocab": list(args[2]), "arities": list(args[3]),
                                    "PAD_ID": int(args[4]),
                                    "precision": int(args[5]) if len(args) > 5
                                    else int(kwargs.get("precision", 4)),
                                    "result": list(out)})
            return out

        return call


def load_dropin():
    """This library's drop-in module (`rpn_cuda_native.py` beside this file)."""
    spec = importlib.util.spec_from_file_location("ws_dropin_rpn_cuda_native",
                                                  os.path.join(_HERE, "rpn_cuda_native.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def load_extension(path: str):
    """A compiled `rpn_cuda_native` extension module from its file."""
    spec = importlib.util.spec_from_file_location("rpn_cuda_native", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def install_native(module, ref_package_dir: str) -> None:
    """Makes `module` the reference's `rpn_cuda_native` and puts the reference package on the
    import path.  Must run before anything imports `warpsymbolic.gpu`."""
    if any(k == "warpsymbolic.gpu" or k.startswith("warpsymbolic.gpu.") for k in sys.modules):
        raise RuntimeError("the reference's gpu package is already imported in this process; "
                           "the native module can only be chosen before that")
    if not os.path.isdir(os.path.join(ref_package_dir, "warpsymbolic")):
        raise FileNotFoundError("no reference package (warpsymbolic/) under %s" % ref_package_dir)
    if ref_package_dir not in sys.path:
        sys.path.insert(0, ref_package_dir)
    sys.modules["rpn_cuda_native"] = module


# ---------------------------------------------------------------------------------------------
# the plain-method workload: 1024 x 2 rows, population 1024, 20 generations, tournament 4
# ---------------------------------------------------------------------------------------------

@dataclass
class PlainMethodConfig:
    """The plain GP method: X 1024×2 fp32 U[-3,3]; y = x0² + 1.5·sin(x1) + N(0, 0.01²);
    population 1024 of at most 30 tokens drawn by the engine's own initialiser, operators
    {+ − × / sin cos exp log sqrt neg} (pow and abs off), 20 generations, tournament 4, fitness
    RMSE; one island, no validation holdout, protected (not strict) evaluation."""
    rows: int = 1024
    pop_size: int = 1024
    max_len: int = 30
    max_constants: int = 10
    generations: int = 20
    tournament: int = 4
    seed: int = 0
    strict: bool = False
    max_time: float = 900.0
    overrides: Dict[str, Any] = field(default_factory=dict)


def plain_method_data(cfg: PlainMethodConfig):
    rng = np.random.default_rng(cfg.seed)
    X = rng.uniform(-3.0, 3.0, size=(cfg.rows, 2)).astype(np.float32)
    noise = rng.normal(0.0, 0.01, size=cfg.rows)
    y = (X[:, 0].astype(np.float64) ** 2 + 1.5 * np.sin(X[:, 1].astype(np.float64))
         + noise).astype(np.float32)
    return X, y


def engine_options(cfg: PlainMethodConfig) -> Dict[str, Any]:
    """`GpuGlobals` settings of the plain-method run (src/warpsymbolic/gpu/config.py)."""
    opts = {
        "USE_OP_POW": False,
        "USE_OP_ABS": False,
        "DEFAULT_TOURNAMENT_SIZE": int(cfg.tournament),
        "FORCE_STRICT_VALIDATION": bool(cfg.strict),
        "USE_INITIAL_POP_CACHE": False,
        "MAX_FORMULA_LENGTH": int(cfg.max_len),
        "GOOD_ENOUGH_RMSE": -1.0,
    }
    opts.update(cfg.overrides)
    return opts


@dataclass
class RunResult:
    formula: Optional[str]
    engine_error: Optional[str]
    generations_run: int
    best_rmse: float
    seconds: float
    generation_seconds: List[float]
    calls: Dict[str, int]
    errors: Dict[str, List[str]]
    native_file: str
    vocab: List[str]


class PlainMethodRunner:
    """Installs `native_module` (wrapped in a RecordingModule) as the reference's extension and
    fits the plain-method workload through `WarpSymbolicRegressor.fit`, as often as asked (the
    estimator reseeds every fit from `random_state`, estimator.py:435-492, so fits repeat)."""

    def __init__(self, native_module, ref_package_dir: str,
                 cfg: Optional[PlainMethodConfig] = None, keep_generations: bool = True):
        self.cfg = cfg or PlainMethodConfig()
        self.native_module = native_module
        self.rec = RecordingModule(native_module, keep_generations=keep_generations)
        install_native(self.rec, ref_package_dir)
        from warpsymbolic.gpu.config import GpuGlobals
        from warpsymbolic.gpu import engine as engine_mod
        from warpsymbolic.api.estimator import WarpSymbolicRegressor
        self._estimator_cls = WarpSymbolicRegressor
        for name, value in engine_options(self.cfg).items():
            if not hasattr(GpuGlobals, name):
                raise ValueError("unknown engine option %s" % name)
            setattr(GpuGlobals, name, value)

        # per-generation wall time: the engine calls evolve_generation_cuda once a generation
        self._stamps: List[float] = []
        self._engine = None
        stamps = self._stamps
        runner = self
        orig = engine_mod.TensorGeneticEngine.evolve_generation_cuda
        orig_run = engine_mod.TensorGeneticEngine.run

        def timed(eng, *a, **k):
            torch.cuda.synchronize()
            stamps.append(time.perf_counter())
            return orig(eng, *a, **k)

        def run_and_keep(eng, *a, **k):
            out = orig_run(eng, *a, **k)
            runner._engine = eng
            return out

        engine_mod.TensorGeneticEngine.evolve_generation_cuda = timed
        engine_mod.TensorGeneticEngine.run = run_and_keep
        self.X, self.y = plain_method_data(self.cfg)

    def reset_records(self) -> None:
        for k in ("calls", "errors"):
            getattr(self.rec, k).clear()
        for k in ("generations", "decodes", "evaluations"):
            del getattr(self.rec, k)[:]

    def fit(self) -> RunResult:
        cfg = self.cfg
        del self._stamps[:]
        self._engine = None
        est = self._estimator_cls(pop_size=cfg.pop_size, n_islands=1, max_len=cfg.max_len,
                                  max_constants=cfg.max_constants, generations=cfg.generations,
                                  validation_fraction=0.0, random_state=cfg.seed, device="cuda",
                                  max_time=cfg.max_time)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        est.fit(self.X, self.y)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        stamps = self._stamps + [t1]
        eng = self._engine
        gens = int(getattr(eng, "last_run_generations", 0)) if eng is not None else 0
        best = float(getattr(eng, "last_run_best_rmse", math.inf)) if eng is not None else math.inf
        vocab = ([eng.grammar.id_to_token[i] for i in sorted(eng.grammar.id_to_token)]
                 if eng is not None else [])
        return RunResult(formula=est.candidate_formula_, engine_error=est.engine_error_,
                         generations_run=gens, best_rmse=best, seconds=t1 - t0,
                         generation_seconds=[b - a for a, b in zip(stamps[:-1], stamps[1:])],
                         calls=dict(self.rec.calls),
                         errors={k: v[:3] for k, v in self.rec.errors.items()},
                         native_file=str(getattr(self.native_module, "__file__", "")),
                         vocab=vocab)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--ref-package", required=True,
                    help="directory holding the reference's warpsymbolic package")
    ap.add_argument("--native", default="dropin",
                    help="'dropin' (this library) or the path of a compiled rpn_cuda_native")
    ap.add_argument("--out", default="", help="write the records here (torch.save)")
    ap.add_argument("--generations", type=int, default=20)
    ap.add_argument("--no-records", action="store_true")
    args = ap.parse_args(argv)
    mod = load_dropin() if args.native == "dropin" else load_extension(args.native)
    cfg = PlainMethodConfig(generations=args.generations)
    runner = PlainMethodRunner(mod, os.path.abspath(args.ref_package), cfg,
                               keep_generations=not args.no_records)
    res = runner.fit()
    rec = runner.rec
    summary = dict(res.__dict__)
    print("REFERENCE_ENGINE_RESULT " + json.dumps(summary))
    if args.out:
        torch.save({"result": summary, "generations": rec.generations, "decodes": rec.decodes,
                    "evaluations": rec.evaluations, "config": cfg.__dict__}, args.out)
    return 0 if res.engine_error is None else 3


if __name__ == "__main__":
    sys.exit(main())
