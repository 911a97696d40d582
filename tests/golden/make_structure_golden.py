"""Generates tests/golden/structure_torch.npz from the REFERENCE's own torch code (CPU).

The reference's Python callers carry CPU-runnable torch formulations of the structure rules next
to the CUDA kernels; this script imports them from src/warpsymbolic/gpu/ and records their
outputs on seeded populations (well-formed programs plus corrupted ones: PAD gaps, leading PADs,
underflows, extra operands, out-of-table tokens):

  valid_clamped    GPUOperators._validate_rpn_batch, torch path      (operators.py:551-570)
  valid_custom     GPUOperators._validate_rpn_batch_custom           (operators.py:660-676)
  valid_stack      GPUSymbolicSimplifier._validate_batch_stack       (gpu_simplifier.py:513-579)
  starts_fallback  GPUOperators._get_subtree_ranges, torch path      (operators.py:912-946)
  tour*_           TensorGeneticEngine.tournament_selection_island, torch path
                   (engine.py:899-966; the candidate matrix is re-drawn from the same seed)

Needs the reference checkout, named by WS_REFERENCE_ROOT; no GPU.
Usage: WS_REFERENCE_ROOT=<checkout> python tests/golden/make_structure_golden.py
"""
from __future__ import annotations

import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("WS_REFERENCE_ROOT") or sys.exit("set WS_REFERENCE_ROOT to the reference checkout")


def random_rows(rng, arity, n, L, pad=0):
    """int64 [n, L]: well-formed programs (left-packed) and corrupted variants."""
    term = [t for t in range(1, len(arity)) if arity[t] == 0]
    un = [t for t in range(1, len(arity)) if arity[t] == 1]
    bi = [t for t in range(1, len(arity)) if arity[t] == 2]
    rows = np.zeros((n, L), dtype=np.int64)
    for b in range(n):
        length = int(rng.integers(1, L + 1))
        seq, depth = [], 0
        while len(seq) < length:
            left = length - len(seq)
            opts = []
            if depth + 1 <= left - 1 or (left == 1 and depth == 0):
                opts.append("t")
            if depth >= 1 and un and left - 1 >= depth - 1:
                opts.append("u")
            if depth >= 2:
                opts.append("b")
            if not opts:
                break
            k = opts[int(rng.integers(len(opts)))]
            if k == "t":
                seq.append(term[int(rng.integers(len(term)))])
                depth += 1
            elif k == "u":
                seq.append(un[int(rng.integers(len(un)))])
            else:
                seq.append(bi[int(rng.integers(len(bi)))])
                depth -= 1
        rows[b, :len(seq)] = seq
        kind = b % 8
        if kind == 1 and len(seq) > 2:  # PAD gap
            rows[b, int(rng.integers(1, len(seq)))] = pad
        elif kind == 2:  # random soup (underflows, extra operands)
            rows[b, :length] = rng.integers(1, len(arity), size=length)
        elif kind == 3:  # leading PAD
            rows[b, 0] = pad
        elif kind == 4 and length < L:  # operand appended after the end
            rows[b, length] = term[0]
        elif kind == 5:  # tokens outside the arity table
            rows[b, int(rng.integers(0, L))] = int(rng.integers(len(arity), 256))
    return rows


def main():
    sys.path.insert(0, os.path.join(REF, "src"))
    from warpsymbolic.gpu.grammar import GPUGrammar, PAD_ID
    from warpsymbolic.gpu.operators import GPUOperators
    from warpsymbolic.gpu.gpu_simplifier import GPUSymbolicSimplifier
    from warpsymbolic.gpu.engine import TensorGeneticEngine

    out = {}
    rng = np.random.default_rng(2024)
    for name, nvars, L, n in (("v3l30", 3, 30, 3000), ("v5l64", 5, 64, 2000)):
        g = GPUGrammar(num_variables=nvars)
        ops = types.SimpleNamespace(
            grammar=g, device=torch.device("cpu"), pop_dtype=torch.uint8,
            terminal_ids=torch.tensor([g.token_to_id[t] for t in g.terminals], dtype=torch.uint8))
        GPUOperators._init_arity_masks(ops)
        simp = types.SimpleNamespace(grammar=g, device=torch.device("cpu"))
        GPUSymbolicSimplifier._build_arity_table(simp)
        ar_ops = ops.token_arity.numpy().astype(np.int32)
        ar_simp = simp.arity_table.numpy().astype(np.int32)
        rows = random_rows(rng, ar_ops, n, L, PAD_ID)
        pop_u8 = torch.from_numpy(rows.astype(np.uint8))
        pop_i64 = torch.from_numpy(rows)
        out[name + "_pop"] = rows.astype(np.uint8)
        out[name + "_arity_ops"] = ar_ops
        out[name + "_arity_simp"] = ar_simp
        out[name + "_valid_clamped"] = GPUOperators._validate_rpn_batch(ops, pop_u8).numpy()
        out[name + "_valid_custom"] = GPUOperators._validate_rpn_batch_custom(
            ops, pop_u8, L).numpy()
        out[name + "_valid_stack"] = GPUSymbolicSimplifier._validate_batch_stack(
            simp, pop_i64).numpy()
        # the torch fallback indexes the table without clamping: rows inside the table only
        inside = np.nonzero((rows < len(ar_ops)).all(axis=1))[0]
        out[name + "_starts_rows"] = inside
        out[name + "_starts_fallback"] = GPUOperators._get_subtree_ranges(
            ops, pop_u8[torch.from_numpy(inside)]).numpy()

    # Island tournament, torch path (the extension loader raises ImportError on this machine).
    eng = types.SimpleNamespace(device=torch.device("cpu"))
    for i, (B, n_isl, T) in enumerate(((4096, 1, 3), (4096, 8, 4), (1000, 10, 7))):
        fit = torch.from_numpy(rng.standard_normal(B).astype(np.float32) ** 2)
        fit[torch.from_numpy(rng.random(B) < 0.02)] = float("nan")
        fit[::97] = fit[0]  # exact ties
        pop = torch.zeros((B, 4), dtype=torch.uint8)
        torch.manual_seed(100 + i)
        win = TensorGeneticEngine.tournament_selection_island(eng, pop, fit, n_isl, T)
        torch.manual_seed(100 + i)
        isz = B // n_isl
        local = torch.randint(0, isz, (n_isl, isz, T))
        cand = (local + torch.arange(0, B, isz).view(n_isl, 1, 1)).view(B, T)
        out["tour%d_fitness" % i] = fit.numpy()
        out["tour%d_cand" % i] = cand.numpy()
        out["tour%d_winner" % i] = win.numpy()
    np.savez_compressed(os.path.join(HERE, "structure_torch.npz"), **out)
    print("wrote", os.path.join(HERE, "structure_torch.npz"))


if __name__ == "__main__":
    main()
