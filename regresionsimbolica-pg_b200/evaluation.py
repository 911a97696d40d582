"""GPUEvaluator -- mirror of src/warpsymbolic/gpu/evaluation.py on libwarpsym.

evaluate_batch keeps the reference's shape heuristics and its two result conventions, but both
run in ONE launch of the fitness pipeline:
  * where the reference would take its fused kernel (RMSE, <= 4 variables, D <= 1024, L <= 256,
    B <= 1.5M; evaluation.py:104-115) the fused kernel's classification is reproduced
    (invalid -> 1e15 / 1e100, per-row metric overflow -> sqrt of that);
  * everywhere else the classic chunked path's classification is reproduced (invalid ->
    INF_VAL, non-finite mean -> sqrt(INF_VAL); evaluation.py:128-198) without materialising
    the [B, D] predictions.
"""
from __future__ import annotations

from typing import Tuple

import torch

from .cuda_vm import CudaRPNVM


class GPUEvaluator:
    FUSED_MAX_BATCH = 1_500_000

    def __init__(self, grammar, device, max_stack=64, dtype=torch.float64, loss_function="RMSE"):
        self.grammar = grammar
        self.device = torch.device(device)
        self.MAX_STACK = max_stack
        self.dtype = dtype
        self.loss_function = loss_function
        self.INF_VAL = 1e15 if dtype == torch.float32 else 1e100
        self._inf_tensor = torch.tensor(self.INF_VAL, device=self.device, dtype=self.dtype)
        self.vm = CudaRPNVM(grammar, self.device)

    def _run_vm(self, population, x, constants=None, strict_mode: int = 0):
        return self.vm.eval(population, x, constants, strict_mode=strict_mode)

    def _normalize_x(self, x: torch.Tensor, y_target: torch.Tensor) -> torch.Tensor:
        """The reference's [Vars, Samples] vs [Samples, Vars] detection (evaluation.py:54-98)."""
        if x.dim() == 1:
            x = x.unsqueeze(0)
        nv = len(self.grammar.active_variables)
        if x.dim() == 2:
            if x.shape[1] == nv and x.shape[0] != nv:
                x = x.T.contiguous()
            elif x.shape[0] == nv and x.shape[1] != nv:
                pass
            elif x.shape[0] == nv and x.shape[1] == nv:
                n = y_target.shape[0]
                if x.shape[1] == n:
                    pass
                elif x.shape[0] == n:
                    x = x.T.contiguous()
            elif x.shape[1] == y_target.shape[0] and x.shape[0] != y_target.shape[0]:
                pass
            elif x.shape[0] == y_target.shape[0] and x.shape[0] != x.shape[1]:
                x = x.T.contiguous()
        return x

    def evaluate_batch(self, population, x, y_target, constants=None, strict_mode: int = 0):
        """Per-program RMSE [B] in self.dtype (evaluation.py:45-198)."""
        if self.loss_function != "RMSE":
            raise NotImplementedError("only the RMSE fitness is implemented on this path")
        B = int(population.shape[0])
        x = self._normalize_x(x, y_target)
        y = y_target.flatten().to(x.dtype)
        fused_semantics = B <= self.FUSED_MAX_BATCH and self.vm.supports_fused_shape(population, x)
        if fused_semantics:
            inv = 1e15 if x.dtype == torch.float32 else 1e100
            out = self.vm.eval_fitness(population, x.contiguous(), constants, y,
                                       strict_mode=strict_mode, policy="fused", loss="rmse",
                                       invalid_value=inv)
        else:
            out = self.vm.eval_fitness(population, x.contiguous(), constants, y,
                                       strict_mode=strict_mode, policy="classic", loss="rmse",
                                       invalid_value=self.INF_VAL)
        return out.to(self.dtype)

    def evaluate_mse(self, population, x, y_target, constants=None, strict_mode: int = 0):
        """Per-program MSE [B] (x dtype) with the classic path's validity rules."""
        x = self._normalize_x(x, y_target)
        return self.vm.eval_fitness(population, x.contiguous(), constants,
                                    y_target.flatten().to(x.dtype), strict_mode=strict_mode,
                                    policy="classic", loss="mse", invalid_value=self.INF_VAL)

    def evaluate_batch_full(self, population, x, y_target, constants=None, strict_mode: int = 0,
                            force_f32: bool = False) -> torch.Tensor:
        """[B, D] absolute errors with INF for invalid programs (evaluation.py:263-334)."""
        B = int(population.shape[0])
        y_flat = y_target.flatten()
        n = y_flat.shape[0]
        if x.dim() == 1:
            x = x.unsqueeze(0)
        if x.dim() == 2 and x.shape[1] != n and x.shape[0] == n:
            x = x.T.contiguous()
        D = int(x.shape[1])
        out_dtype = torch.float32 if force_f32 else self.dtype
        inf_out = 1e20 if force_f32 else self.INF_VAL
        out = torch.full((B, D), inf_out, device=self.device, dtype=out_dtype)
        target = y_flat.unsqueeze(0)
        step = 100000
        for i in range(0, B, step):
            j = min(B, i + step)
            sub_c = constants[i:j] if constants is not None else None
            preds, sp, err = self._run_vm(population[i:j], x, sub_c, strict_mode=strict_mode)
            valid = (sp == 1) & (err == 0) & ~torch.isnan(preds) & ~torch.isinf(preds)
            preds = torch.where(valid, preds, torch.zeros_like(preds))
            ind_valid = valid.view(j - i, D).all(dim=1).unsqueeze(1).expand(j - i, D)
            ae = torch.abs(preds.view(j - i, D) - target)
            ae = torch.where(torch.isnan(ae) | torch.isinf(ae) | ~ind_valid,
                             torch.tensor(inf_out, device=self.device, dtype=out_dtype),
                             ae.to(out_dtype))
            out[i:j] = ae
        return out

    def validate_strict(self, population, x, y_target, constants=None) -> dict:
        """Strict-math validation (evaluation.py:336-402): per program the number of rows with a
        domain error / bad stack / non-finite prediction, and the RMSE of valid programs."""
        x = self._normalize_x(x, y_target)
        B = int(population.shape[0])
        D = int(x.shape[1])
        ninv = torch.empty(B, dtype=torch.int32, device=self.device)
        sse = self.vm.eval_fitness(population, x.contiguous(), constants,
                                   y_target.flatten().to(x.dtype), strict_mode=1,
                                   policy="classic", loss="sse", invalid_value=float("inf"),
                                   out_ninvalid=ninv)
        n_errors = ninv.to(torch.int64)
        mse = (sse / D).to(x.dtype)
        rmse = torch.sqrt(mse).to(self.dtype)
        rmse = torch.where(n_errors > 0, self._inf_tensor, rmse)
        return {"rmse": rmse, "n_errors": n_errors, "n_total": D, "is_valid": n_errors == 0}
