"""Many problems in one launch sequence, CUDA-graph replay, and a schedule autotuner.

A genetic-programming run on many datasets (one population per problem) scores every problem's
population each generation.  The reference does that one `evaluate_batch` call per problem
(evaluation.py:45-198).  Here all problems go through ONE compile launch, ONE length sort and ONE
persistent evaluator launch (libwarpsym's ws_batch_*), so small problems do not leave the GPU
idle and the launch count does not grow with the number of problems:

    problems = [BatchProblem(pop_p, x_p, y_p, consts_p, grammar_p) for p in ...]
    bf = BatchedFitness(problems, loss="mse", policy="classic")
    bf.evaluate()                       # bf.outputs[p]: [B_p] losses of problem p
    graph = bf.capture()                # compile + sort + evaluate as one CUDA graph
    ... rewrite populations / constants in place ...
    graph.replay()                      # bf.outputs hold the new losses

`autotune(problems, ...)` times every compiled tile schedule (rows per lane x warps x programs
per block x shared-memory budget) on the batch and returns the fastest; results are cached per
shape signature.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import torch

from . import _native as N
from ._tensors import check_cuda, dtype_code, ptr, stream_of
from .grammar import PI_VAL, E_VAL

_POLICIES = {"fused": N.WS_POLICY_FUSED, "classic": N.WS_POLICY_CLASSIC}
_LOSSES = {"rmse": N.WS_LOSS_RMSE, "mse": N.WS_LOSS_MSE, "r2": N.WS_LOSS_R2, "sse": N.WS_LOSS_SSE}


@dataclass
class BatchProblem:
    population: torch.Tensor            # [B, L] uint8 (all problems share L)
    x: torch.Tensor                     # [V, D]
    y: torch.Tensor                     # [D]
    constants: Optional[torch.Tensor]   # [B, K] or None
    grammar: object                     # GPUGrammar of this problem (token IDs)


class BatchedFitness:
    """Per-program losses of many problems from one launch sequence.  The plan (and the
    device descriptors it writes on the current stream) fixes every tensor's address and shape:
    rewrite populations and constants in place between calls, never reallocate them."""

    def __init__(self, problems: Sequence[BatchProblem], *, loss: str = "mse",
                 policy: str = "classic", strict_mode: int = 0, schedule: int = 0,
                 invalid_value: Optional[float] = None, count_invalid: bool = False,
                 workspace: Optional[Callable[[int], torch.Tensor]] = None):
        """`workspace`, when given, returns a uint8 device tensor of at least the requested
        bytes (256-byte aligned); a caller that replans often passes one buffer it reuses
        instead of an allocation per plan (work on one stream is ordered, so a new plan may take
        over memory that queued work of an older plan still uses)."""
        if not problems:
            raise ValueError("no problems")
        self.problems = list(problems)
        L = int(self.problems[0].population.shape[1])
        dtype = self.problems[0].x.dtype
        self.device = self.problems[0].x.device
        code = dtype_code(dtype)
        lk = _LOSSES[loss]
        out_dtype = torch.float64 if lk == N.WS_LOSS_SSE else dtype
        if invalid_value is None:
            invalid_value = 1e15 if dtype == torch.float32 else 1e100
        self._opts = N.FitnessOpts(int(strict_mode), _POLICIES[policy], lk, int(schedule),
                                   float(invalid_value), 0, 0)
        arr = (N.Problem * len(self.problems))()
        self._keep: List[object] = []   # tensors and token maps referenced by the descriptors
        # outputs of all problems are views of one flat buffer (one copy reads them all back)
        total = sum(int(p.population.shape[0]) for p in self.problems)
        self.flat_out = torch.empty(max(total, 1), dtype=out_dtype, device=self.device)
        self.flat_ninvalid = (torch.empty(max(total, 1), dtype=torch.int32, device=self.device)
                              if count_invalid else None)
        self.outputs: List[torch.Tensor] = []
        self.ninvalid: List[Optional[torch.Tensor]] = []
        off = 0
        for i, p in enumerate(self.problems):
            pop, x, y = p.population, p.x, p.y.reshape(-1)
            for t, nm in ((pop, "population"), (x, "x"), (y, "y")):
                check_cuda(t, "problem %d %s" % (i, nm))
            if pop.dtype != torch.uint8 or pop.dim() != 2 or int(pop.shape[1]) != L:
                raise RuntimeError("problem %d: population must be uint8 [B, %d]" % (i, L))
            if x.dtype != dtype or y.dtype != dtype:
                raise RuntimeError("problem %d: x and y must be %s" % (i, dtype))
            B = int(pop.shape[0])
            V, D = int(x.shape[0]), int(x.shape[1])
            if y.numel() != D:
                raise RuntimeError("problem %d: y must have shape [D]" % i)
            c = p.constants
            K = 0
            if c is not None and c.numel() > 0:
                check_cuda(c, "problem %d constants" % i)
                if c.dtype != dtype or c.dim() != 2 or int(c.shape[0]) != B:
                    raise RuntimeError("problem %d: constants must be %s [B, K]" % (i, dtype))
                K = int(c.shape[1])
            out = self.flat_out[off:off + B]
            nin = self.flat_ninvalid[off:off + B] if count_invalid else None
            off += B
            tmap = N.TokenMap.from_args(*p.grammar.scalar_ids(), pi_val=PI_VAL, e_val=E_VAL)
            self._keep += [pop, x, y, c, out, nin, tmap]
            self.outputs.append(out)
            self.ninvalid.append(nin)
            arr[i] = N.Problem(ptr(pop), B, ptr(x), V, D, ptr(c) if K > 0 else None, K, ptr(y),
                               ptr(out), ptr(nin), C.pointer(tmap))
        self._arr = arr
        lib = N.lib()
        need = C.c_size_t(0)
        N.check(lib.ws_batch_workspace_bytes(code, C.cast(arr, C.c_void_p), len(arr), L,
                                             C.byref(self._opts), C.byref(need)))
        nbytes = max(int(need.value), 256)
        self.workspace = (workspace(nbytes) if workspace is not None else
                          torch.empty(nbytes, dtype=torch.uint8, device=self.device))
        h = C.c_void_p()
        N.check(lib.ws_batch_create(code, C.cast(arr, C.c_void_p), len(arr), L,
                                    C.byref(self._opts), ptr(self.workspace),
                                    int(self.workspace.numel()), stream_of(self.workspace),
                                    C.byref(h)))
        self._h = h
        self.L = L

    # -- launches ---------------------------------------------------------------------------
    def evaluate(self, phase: int = 0, stream=None) -> List[torch.Tensor]:
        """Launches compile + sort + evaluate (or one phase) on `stream` (default: the current
        stream); returns the per-problem output tensors (written asynchronously)."""
        if self._h is None:
            raise RuntimeError("batch is closed")
        st = C.c_void_p(stream.cuda_stream) if stream is not None else stream_of(self.workspace)
        N.check(N.lib().ws_batch_eval(self._h, int(phase), st))
        return self.outputs

    def capture(self, warmup: int = 1) -> torch.cuda.CUDAGraph:
        """Captures one evaluate() into a CUDA graph (after `warmup` eager runs on a side
        stream, as graph capture requires)."""
        s = torch.cuda.Stream(device=self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            for _ in range(warmup):
                self.evaluate(stream=s)
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.evaluate()
        return g

    def set_cancel_flag(self, flag: Optional[torch.Tensor]) -> None:
        """Attaches a one-element int32 device tensor (None detaches): while it holds a nonzero
        value, a launch takes no further work items and its outputs are incomplete (the caller
        discards them); see ws_batch_set_cancel."""
        if flag is not None and (flag.dtype != torch.int32 or flag.device != self.device
                                 or flag.numel() != 1):
            raise ValueError("the cancel flag is a one-element int32 tensor on the batch's device")
        self._cancel = flag  # kept alive while attached
        N.check(N.lib().ws_batch_set_cancel(self._h, ptr(flag) if flag is not None else None))

    def info(self) -> Dict[str, int]:
        lib = N.lib()
        keys = ("work_items", "rows_per_lane", "programs_per_block", "smem_bytes", "resident_ctas",
                "programs")
        return {k: int(lib.ws_batch_info(self._h, i)) for i, k in enumerate(keys)}

    def close(self) -> None:
        if getattr(self, "_h", None) is not None:
            N.lib().ws_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- autotuner ---------------------------------------------------------------------------
_TUNED: Dict[Tuple, int] = {}


def signature(problems: Sequence[BatchProblem], loss: str, policy: str, strict_mode: int) -> Tuple:
    """Shape class of a batch: dtype, L, loss/policy/mode, problem count, and the programs, rows
    and variables of its problems bucketed (rows and programs to powers of two)."""
    def b2(v):
        return int(v).bit_length()
    p0 = problems[0]
    shapes = sorted((b2(p.population.shape[0]), b2(p.x.shape[1]), int(p.x.shape[0]))
                    for p in problems)
    return (str(p0.x.dtype), int(p0.population.shape[1]), loss, policy, int(strict_mode),
            len(problems), tuple(shapes))


def autotune(problems: Sequence[BatchProblem], *, loss: str = "mse", policy: str = "classic",
             strict_mode: int = 0, schedules: Optional[Sequence[int]] = None, reps: int = 3,
             use_cache: bool = True) -> Tuple[int, Dict[int, float]]:
    """Times the evaluator launch of every compiled schedule on this batch (CUDA events, after
    one warm-up) and returns (fastest schedule, {schedule: ms}).  Schedules that cannot run the
    batch (shared-memory limits) are skipped."""
    key = signature(problems, loss, policy, strict_mode)
    if use_cache and key in _TUNED:
        return _TUNED[key], {}
    if schedules is None:
        schedules = range(1, int(N.lib().ws_schedule_count()))
    times: Dict[int, float] = {}
    for s in schedules:
        try:
            bf = BatchedFitness(problems, loss=loss, policy=policy, strict_mode=strict_mode,
                                schedule=int(s))
        except RuntimeError:
            continue
        try:
            bf.evaluate(phase=N.WS_PHASE_COMPILE)
            bf.evaluate(phase=N.WS_PHASE_EVALUATE)
            best = float("inf")
            for _ in range(reps):
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record()
                bf.evaluate(phase=N.WS_PHASE_EVALUATE)
                b.record()
                b.synchronize()
                best = min(best, a.elapsed_time(b))
            times[int(s)] = best
        finally:
            bf.close()
    if not times:
        raise RuntimeError("no schedule can run this batch")
    best_s = min(times, key=times.get)
    _TUNED[key] = best_s
    return best_s, times
