"""Device-side genetic-programming generations for many problems at once (libwarpsym ws_gp_*).

    gp = GPStep(problems, fitness, seeds, tournament_size=3, crossover_rate=0.7, ...)
    gp.step()              # populations and constants of every problem become the next generation

`problems` are the same BatchProblem records the batched evaluator uses (their population and
constants tensors are rewritten in place, so a BatchedFitness over them sees every new
generation without re-planning); `fitness[p]` is problem p's [B] loss tensor (lower is better),
e.g. BatchedFitness.outputs.  A generation is three launches; the generation counters live on
the device (one per problem, starting at `generations[p]`), so evaluate + step can be captured
once as a CUDA graph and replayed per generation.
Offspring of a problem depend only on its seed, the generation and its own population and
fitness -- never on the other problems of the launch.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, List, Optional, Sequence

import torch

from . import _native as N
from ._tensors import check_cuda, dtype_code, ptr, stream_of
from .grammar import PI_VAL, E_VAL


class GPStep:
    def __init__(self, problems: Sequence, fitness: Sequence[torch.Tensor], seeds: Sequence[int],
                 *, generations: Optional[Sequence[int]] = None, tournament_size: int = 3,
                 elitism: bool = True, crossover_rate: float = 0.7,
                 mutation_rate: float = 0.05, const_mutation_rate: float = 0.1,
                 const_sigma: float = 0.1, parsimony_eps: float = 1e-9,
                 workspace: Optional[Callable[[int], torch.Tensor]] = None):
        if not problems:
            raise ValueError("no problems")
        if len(fitness) != len(problems) or len(seeds) != len(problems):
            raise ValueError("one fitness tensor and one seed per problem")
        if generations is None:
            generations = [0] * len(problems)
        if len(generations) != len(problems):
            raise ValueError("one starting generation per problem")
        L = int(problems[0].population.shape[1])
        dtype = fitness[0].dtype
        code = dtype_code(dtype)
        arr = (N.GpProblem * len(problems))()
        self._keep: List[object] = []
        for i, (p, f, s) in enumerate(zip(problems, fitness, seeds)):
            check_cuda(p.population, "problem %d population" % i)
            check_cuda(f, "problem %d fitness" % i)
            B = int(p.population.shape[0])
            if int(p.population.shape[1]) != L or p.population.dtype != torch.uint8:
                raise RuntimeError("problem %d: population must be uint8 [B, %d]" % (i, L))
            if f.dtype != dtype or f.numel() != B:
                raise RuntimeError("problem %d: fitness must be %s [B]" % (i, dtype))
            c = p.constants
            K = 0
            if c is not None and c.numel() > 0:
                check_cuda(c, "problem %d constants" % i)
                if c.dtype != dtype or int(c.shape[0]) != B:
                    raise RuntimeError("problem %d: constants must be %s [B, K]" % (i, dtype))
                K = int(c.shape[1])
            tmap = N.TokenMap.from_args(*p.grammar.scalar_ids(), pi_val=PI_VAL, e_val=E_VAL)
            self._keep += [p.population, c, f, tmap]
            arr[i] = N.GpProblem(ptr(p.population), B, ptr(c) if K > 0 else None, K, ptr(f),
                                 len(p.grammar.active_variables), C.pointer(tmap),
                                 int(s) & 0xFFFFFFFFFFFFFFFF, int(generations[i]))
        self._arr = arr
        self._opts = N.GpOpts(int(tournament_size), 1 if elitism else 0, float(crossover_rate),
                              float(mutation_rate), float(const_mutation_rate), float(const_sigma),
                              float(parsimony_eps), 0)
        lib = N.lib()
        need = C.c_size_t(0)
        N.check(lib.ws_gp_workspace_bytes(code, C.cast(arr, C.c_void_p), len(arr), L, C.byref(need)))
        self.device = problems[0].population.device
        nbytes = max(int(need.value), 256)
        self.workspace = (workspace(nbytes) if workspace is not None else
                          torch.empty(nbytes, dtype=torch.uint8, device=self.device))
        h = C.c_void_p()
        N.check(lib.ws_gp_create(code, C.cast(arr, C.c_void_p), len(arr), L, C.byref(self._opts),
                                 ptr(self.workspace), int(self.workspace.numel()),
                                 stream_of(self.workspace), C.byref(h)))
        self._h = h

    def step(self, stream=None) -> None:
        st = C.c_void_p(stream.cuda_stream) if stream is not None else stream_of(self.workspace)
        N.check(N.lib().ws_gp_step(self._h, st))

    def set_generation(self, generation: int, stream=None) -> None:
        st = C.c_void_p(stream.cuda_stream) if stream is not None else stream_of(self.workspace)
        N.check(N.lib().ws_gp_set_generation(self._h, int(generation), st))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None:
            N.lib().ws_gp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
