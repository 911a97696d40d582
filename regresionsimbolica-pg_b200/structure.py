"""Population-structure operations on the GPU: stack validation, subtree starts, tournament
selection.  Mirrors the reference's Python callers of these kernels, with one entry per rule the
reference applies:

  validate_population(..., rule="kernel")   GPUOperators._validate_rpn_batch, CUDA path
                                            (gpu/operators.py:535-549 -> rpn_kernels.cu:850-900)
  validate_population(..., rule="clamped")  its torch fallback and _validate_rpn_batch_custom
                                            (gpu/operators.py:551-570, 660-676)
  validate_population(..., rule="stack")    GPUSymbolicSimplifier._validate_batch_stack
                                            (gpu/gpu_simplifier.py:513-579)
  subtree_starts(...)                       GPUOperators._get_subtree_ranges, CUDA path
                                            (gpu/operators.py:891-910 -> rpn_kernels.cu:433-504)
  simplifier_subtree_starts(...)            precompute_subtree_starts (simplify_kernels.cu:612)
  tournament_selection_island(...)          TensorGeneticEngine.tournament_selection_island
                                            (gpu/engine.py:899-966)

Every function runs the sm_100a kernels of libwarpsym.so; there is no CPU path.
"""
from __future__ import annotations

import torch

from . import _native as N
from ._tensors import check_cuda, ptr, stream_of

_RULES = {"kernel": N.WS_VALIDATE_KERNEL, "clamped": N.WS_VALIDATE_CLAMPED,
          "stack": N.WS_VALIDATE_STACK}


def _arity_i32(token_arity: torch.Tensor, device) -> torch.Tensor:
    return token_arity.to(device=device, dtype=torch.int32).contiguous()


def validate_population(population: torch.Tensor, token_arity: torch.Tensor, pad_id: int = 0,
                        rule: str = "kernel", out: torch.Tensor | None = None) -> torch.Tensor:
    """bool [B]: True where the program's stack discipline is valid under `rule`.
    population: uint8 or int64 [B, L] on a CUDA device; token_arity: arity per token value."""
    check_cuda(population, "population")
    if population.dtype not in (torch.uint8, torch.int64):
        raise RuntimeError("population must hold uint8 or int64 tokens")
    if rule not in _RULES:
        raise ValueError("rule must be one of %s" % sorted(_RULES))
    B, L = int(population.size(0)), int(population.size(1))
    ar = _arity_i32(token_arity, population.device)
    if out is None:
        out = torch.empty(B, dtype=torch.bool, device=population.device)
    N.check(N.lib().ws_validate_rpn_batch(ptr(population), population.element_size(), B, L,
                                          ptr(ar), int(ar.numel()), int(pad_id), _RULES[rule],
                                          ptr(out), stream_of(population)))
    return out


def subtree_starts(population: torch.Tensor, token_arity: torch.Tensor, pad_id: int = 0,
                   with_lengths: bool = False):
    """int64 [B, L]: start of the subtree that ends at each position (-1 for PAD and for
    operators with missing operands); with_lengths also returns int64 [B] (first PAD, else L)."""
    check_cuda(population, "population")
    if population.dtype != torch.uint8:
        raise RuntimeError("population must hold uint8 tokens")
    B, L = int(population.size(0)), int(population.size(1))
    ar = _arity_i32(token_arity, population.device)
    starts = torch.empty((B, L), dtype=torch.int64, device=population.device)
    lengths = torch.empty(B, dtype=torch.int64, device=population.device) if with_lengths else None
    N.check(N.lib().ws_find_subtree_ranges(ptr(population), B, L, ptr(ar), int(ar.numel()),
                                           int(pad_id), ptr(starts), ptr(lengths),
                                           stream_of(population)))
    return (starts, lengths) if with_lengths else starts


def simplifier_subtree_starts(population: torch.Tensor, arity_table: torch.Tensor) -> torch.Tensor:
    """int64 [B, L] by the simplifier's forward recurrence (simplify_kernels.cu:612-661)."""
    check_cuda(population, "population")
    pop = population if population.dtype == torch.int64 else population.to(torch.int64)
    pop = pop.contiguous()
    B, L = int(pop.size(0)), int(pop.size(1))
    ar = _arity_i32(arity_table, pop.device)
    out = torch.empty((B, L), dtype=torch.int64, device=pop.device)
    N.check(N.lib().ws_precompute_subtree_starts(ptr(pop), B, L, ptr(ar), int(ar.numel()),
                                                 ptr(out), stream_of(pop)))
    return out


def tournament_select(fitness: torch.Tensor, candidates: torch.Tensor, *,
                      errors: torch.Tensor | None = None, cases: torch.Tensor | None = None,
                      lengths: torch.Tensor | None = None, mad_eps: torch.Tensor | None = None,
                      island_size: int = 0, n_islands: int = 1) -> torch.Tensor:
    """int64 [B] winners.  candidates: int64 [B, T] global indices, or int32 [B, T] offsets
    (reduced into the slot's island: base + offset % span, the evolve_generation form)."""
    check_cuda(fitness, "fitness")
    check_cuda(candidates, "candidates")
    fit = fitness.to(torch.float32).contiguous()
    B, T = int(fit.numel()), int(candidates.size(1))
    out = torch.empty(B, dtype=torch.int64, device=fit.device)

    def opt(t, dt):
        if t is None or t.numel() == 0:
            return None
        return t.to(device=fit.device, dtype=dt).contiguous()

    errors, cases = opt(errors, torch.float32), opt(cases, torch.int32)
    lengths, mad_eps = opt(lengths, torch.float32), opt(mad_eps, torch.float32)
    n_data = int(errors.size(1)) if errors is not None else 0
    lib = N.lib()
    if candidates.dtype == torch.int64:
        N.check(lib.ws_tournament_select(ptr(fit), B, ptr(errors), n_data, ptr(candidates), T,
                                         ptr(cases), ptr(lengths), ptr(mad_eps), ptr(out),
                                         stream_of(fit)))
    elif candidates.dtype == torch.int32:
        N.check(lib.ws_tournament_select_offsets(ptr(fit), B, ptr(errors), n_data,
                                                 ptr(candidates), T, ptr(cases), ptr(lengths),
                                                 ptr(mad_eps), int(island_size), int(n_islands),
                                                 ptr(out), stream_of(fit)))
    else:
        raise RuntimeError("candidates must be int64 indices or int32 offsets")
    return out


def tournament_selection_island(fitness: torch.Tensor, n_islands: int, tournament_size: int = 3,
                                generator: torch.Generator | None = None) -> torch.Tensor:
    """Island tournament of the engine (engine.py:899-966): NaN fitness counts as +inf, each
    slot draws tournament_size local indices in its own island, the smallest fitness wins."""
    B = int(fitness.numel())
    if B % n_islands != 0:
        raise ValueError(f"Population {B} not divisible by islands {n_islands}")
    island_size = B // n_islands
    fit = torch.nan_to_num(fitness, nan=float("inf"))
    local = torch.randint(0, island_size, (n_islands, island_size, tournament_size),
                          device=fit.device, generator=generator)
    offsets = torch.arange(0, B, island_size, device=fit.device).view(n_islands, 1, 1)
    cand = (local + offsets).view(B, tournament_size).contiguous()
    return tournament_select(fit, cand)
