"""GPUSymbolicSimplifier mirror (src/warpsymbolic/gpu/gpu_simplifier.py:27-439): the tables the
reference builds from the grammar (arity table, literal values, literal IDs, operator IDs with
their aliases) and its simplify_batch wrapper around the kernel: rows holding a free constant
C are left byte-for-byte unchanged (constant slots are positional), the kernel rewrites the
others, and rows it leaves stack-invalid are restored (the simplifier's own validity rule,
gpu_simplifier.py:513-579).  The reference's torch rewrite passes, used there for programs
longer than 256 tokens or when the extension is missing, are not part of this library: such
programs are returned unchanged.
"""
from __future__ import annotations

import math
from typing import Optional, Tuple

import torch

from . import rpn_cuda_native as _rcn
from .grammar import OPERATORS, PAD_ID
from .structure import validate_population


def _is_number(t: str) -> bool:
    return t.replace('.', '', 1).isdigit() or (t.startswith('-') and
                                                t[1:].replace('.', '', 1).isdigit())


class GPUSymbolicSimplifier:
    def __init__(self, grammar, device):
        self.grammar = grammar
        self.device = torch.device(device)
        g = grammar

        def first(names):
            for n in names:
                if n in g.token_to_id:
                    return g.token_to_id[n]
            return -1

        max_id = max(max(g.id_to_token.keys()) + 1, PAD_ID + 1)
        ar = torch.zeros(max_id, dtype=torch.int32)
        for tok, tid in g.token_to_id.items():
            ar[tid] = OPERATORS.get(tok, 0)
        for alias in ('fact', 'factorial'):
            if alias in g.token_to_id:
                ar[g.token_to_id[alias]] = 1
        self.arity_table = ar.to(self.device)
        vt = torch.full((max_id,), float('nan'), dtype=torch.float32)
        for tok, tid in g.token_to_id.items():
            if _is_number(tok):
                vt[tid] = float(tok)
            elif tok == 'pi':
                vt[tid] = float(math.pi)
            elif tok == 'e':
                vt[tid] = float(math.e)
        self.val_table = vt.to(self.device)
        lits = [g.token_to_id[t] for t in g.terminals if _is_number(t)]
        self.literal_ids = torch.tensor(lits, dtype=torch.int64, device=self.device)
        self.literal_vals = torch.tensor([float(g.id_to_token[i]) for i in lits],
                                         dtype=torch.float32, device=self.device)
        self.op_ids = (
            g.token_to_id.get('+', -1), g.token_to_id.get('-', -1), g.token_to_id.get('*', -1),
            g.token_to_id.get('/', -1), first(['neg']), first(['%', 'mod']),
            first(['pow', '^', '**']), g.token_to_id.get('sin', -1),
            g.token_to_id.get('cos', -1), g.token_to_id.get('tan', -1),
            g.token_to_id.get('asin', -1), g.token_to_id.get('acos', -1),
            g.token_to_id.get('atan', -1), first(['log', 'ln']), first(['exp']),
            first(['sqrt']), first(['abs']), first(['gamma', '!']),
            first(['lgamma', 'lg', 'g']), first(['floor', '_']), g.token_to_id.get('ceil', -1),
            g.token_to_id.get('sign', -1), first(['0', '0.0']), first(['1', '1.0']),
            first(['2', '2.0']), g.token_to_id.get('3', -1), g.token_to_id.get('4', -1),
            g.token_to_id.get('5', -1), g.token_to_id.get('6', -1))

    def simplify_batch(self, population: torch.Tensor, constants: Optional[torch.Tensor] = None,
                       max_passes: int = 3) -> Tuple[torch.Tensor, Optional[torch.Tensor], int]:
        """(simplified population, constants, 0), as the reference's CUDA path returns."""
        B, L = population.shape
        c_id = self.grammar.token_to_id.get('C', -1)
        if c_id >= 0:
            free = (population == c_id).any(dim=1)
            if bool(free.any()):
                eligible = ~free
                if not bool(eligible.any()):
                    return population.clone(), constants, 0
                sub, sub_c, n = self.simplify_batch(
                    population[eligible],
                    constants[eligible] if constants is not None else None, max_passes)
                out = population.clone()
                out[eligible] = sub
                if constants is None:
                    return out, None, n
                out_c = constants.clone()
                out_c[eligible] = sub_c
                return out, out_c, n
        pop = population.clone()
        if L > 256:
            return pop, constants, 0
        work = pop.to(torch.int64).contiguous()
        _rcn.simplify_batch(work, self.arity_table, self.val_table, self.literal_ids,
                            self.literal_vals, max_passes, *self.op_ids)
        work = work.to(pop.dtype)
        ok = validate_population(work, self.arity_table, PAD_ID, "stack")
        work[~ok] = population[~ok]
        return work, constants, 0
