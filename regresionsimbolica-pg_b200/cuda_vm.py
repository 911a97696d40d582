"""CudaRPNVM -- mirror of src/warpsymbolic/gpu/cuda_vm.py on top of libwarpsym.

Keeps the reference's interface (eval, eval_fused, _launch_fused, supports_fused_shape and the
fused-envelope limits) and adds eval_fitness, the envelope-free evaluator behind
GPUEvaluator.evaluate_batch.  The reference's block/warp autotune (cuda_vm.py:190-242) is
replaced by the schedule choice inside libwarpsym; `last_eval_mode` reports "fitness".
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import torch

from . import _native as N
from ._tensors import check_cuda, dtype_code, ptr, stream_of, workspace
from .grammar import PI_VAL, E_VAL

_POLICIES = {"fused": N.WS_POLICY_FUSED, "classic": N.WS_POLICY_CLASSIC}
_LOSSES = {"rmse": N.WS_LOSS_RMSE, "mse": N.WS_LOSS_MSE, "r2": N.WS_LOSS_R2, "sse": N.WS_LOSS_SSE}


class CudaRPNVM:
    FUSED_MAX_VARS = 4
    FUSED_MAX_L = 256
    FUSED_MAX_D = 1024

    def __init__(self, grammar, device):
        self.grammar = grammar
        self.device = torch.device(device)
        self._cache_ids()
        self._output_cache = {}
        self._empty_constants_cache = {}
        self.last_eval_mode = "fitness"

    def _cache_ids(self):
        self.ids = self.grammar.scalar_ids()
        self.num_vars = len(self.grammar.active_variables)
        self._tmap = N.TokenMap.from_args(*self.ids, pi_val=PI_VAL, e_val=E_VAL)

    def token_map(self) -> N.TokenMap:
        return self._tmap

    def _constants(self, constants, B, dtype):
        if constants is None:
            key = (B, dtype)
            if key not in self._empty_constants_cache:
                self._empty_constants_cache[key] = torch.empty((B, 0), device=self.device, dtype=dtype)
            return self._empty_constants_cache[key]
        if not constants.is_contiguous():
            constants = constants.contiguous()
        if constants.dtype != dtype:
            constants = constants.to(dtype)
        return constants

    # ---- classic path (cuda_vm.py:84-152) ----------------------------------------------------
    def eval(self, population, x, constants, strict_mode: int = 0) -> Tuple[torch.Tensor, ...]:
        """Returns (preds [B, D], sp [B, D], error [B, D]); buffers are reused per (B, D, dtype)
        as in the reference, so callers must clone results they keep."""
        B = int(population.shape[0])
        _, D = x.shape
        population = population.contiguous()
        x = x.contiguous()
        dtype = x.dtype
        constants = self._constants(constants, B, dtype)
        key = (B, int(D), dtype)
        if key not in self._output_cache:
            self._output_cache[key] = (
                torch.empty((B, D), dtype=dtype, device=self.device),
                torch.empty((B, D), dtype=torch.int32, device=self.device),
                torch.empty((B, D), dtype=torch.uint8, device=self.device))
        out_preds, out_sp, out_error = self._output_cache[key]
        from .rpn_cuda_native import eval_rpn
        eval_rpn(population, x, constants, out_preds, out_sp, out_error, *self.ids,
                 PI_VAL, E_VAL, strict_mode)
        return out_preds, out_sp, out_error

    # ---- fused path (cuda_vm.py:154-296) -----------------------------------------------------
    def _launch_fused(self, population, x, constants, y_target, out_rmse, strict_mode, launch_mode):
        if x.ndim != 2 or int(x.shape[0]) != self.num_vars:
            raise ValueError("x must have shape [%d, D] for this grammar" % self.num_vars)
        from .rpn_cuda_native import eval_rpn_fused
        eval_rpn_fused(population, x, constants, y_target, out_rmse, *self.ids, PI_VAL, E_VAL,
                       strict_mode, launch_mode)

    def supports_fused_shape(self, population, x) -> bool:
        if population.ndim != 2 or x.ndim != 2:
            return False
        return (int(population.shape[0]) > 0 and int(population.shape[1]) > 0
                and 0 < self.num_vars <= self.FUSED_MAX_VARS
                and int(x.shape[0]) == self.num_vars and int(x.shape[1]) > 0
                and int(population.shape[1]) <= self.FUSED_MAX_L
                and int(x.shape[1]) <= self.FUSED_MAX_D)

    def eval_fused(self, population, x, constants, y_target, strict_mode: int = 0):
        if not self.supports_fused_shape(population, x):
            raise ValueError(
                "eval_rpn_fused only supports at most %d variables, programs of length %d, and "
                "%d samples; use eval() for the classic safe path."
                % (self.FUSED_MAX_VARS, self.FUSED_MAX_L, self.FUSED_MAX_D))
        B = int(population.shape[0])
        dtype = x.dtype
        population, x, y_target = population.contiguous(), x.contiguous(), y_target.contiguous()
        constants = self._constants(constants, B, dtype)
        key = ("fused", B, dtype)
        if key not in self._output_cache:
            self._output_cache[key] = torch.empty(B, dtype=dtype, device=self.device)
        out_rmse = self._output_cache[key]
        self.last_eval_mode = "fitness"
        self._launch_fused(population, x, constants, y_target, out_rmse, strict_mode, 0)
        return out_rmse

    # ---- envelope-free fitness (new) -------------------------------------------------------------
    def eval_fitness(self, population, x, constants, y_target, *, strict_mode: int = 0,
                     policy: str = "fused", loss: str = "rmse",
                     invalid_value: Optional[float] = None, out: Optional[torch.Tensor] = None,
                     out_ninvalid: Optional[torch.Tensor] = None, schedule: int = 0,
                     stream=None, phase: int = 0, workspace_tensor=None) -> torch.Tensor:
        """Per-program loss of every program on (x [V, D], y [D]) in one pipeline, any V <= 64,
        any D, L <= 256.  policy "fused" reproduces rpn_eval_fused_kernel's classification,
        "classic" the chunked evaluate_batch path.  Returns `out` ([B], x dtype; float64 for
        loss="sse")."""
        check_cuda(population, "population")
        check_cuda(x, "x")
        check_cuda(y_target, "y_target")
        if population.dtype != torch.uint8 or population.dim() != 2:
            raise RuntimeError("population must be uint8 [B, L]")
        B, L = int(population.shape[0]), int(population.shape[1])
        V, D = int(x.shape[0]), int(x.shape[1])
        if y_target.numel() != D:
            raise RuntimeError("y_target must have shape [D]")
        dtype = x.dtype
        code = dtype_code(dtype)
        y_target = y_target.reshape(-1)
        if y_target.dtype != dtype:
            y_target = y_target.to(dtype)
        constants = self._constants(constants, B, dtype)
        K = int(constants.shape[1]) if constants.dim() > 1 else 0
        if K > 0:
            check_cuda(constants, "constants")
        lk = _LOSSES[loss]
        out_dtype = torch.float64 if lk == N.WS_LOSS_SSE else dtype
        if out is None:
            out = torch.empty(B, dtype=out_dtype, device=x.device)
        elif out.dtype != out_dtype or out.numel() != B or not out.is_contiguous():
            raise RuntimeError("out must be a contiguous [B] %s tensor" % out_dtype)
        if out_ninvalid is not None and (out_ninvalid.dtype != torch.int32 or out_ninvalid.numel() != B):
            raise RuntimeError("out_ninvalid must be a [B] int32 tensor")
        if invalid_value is None:
            invalid_value = 1e15 if dtype == torch.float32 else 1e100
        opts = N.FitnessOpts(int(strict_mode), _POLICIES[policy], lk, int(schedule),
                             float(invalid_value), int(phase), 0)
        lib = N.lib()
        nbytes = lib.ws_fitness_workspace_bytes(B, L, code)
        if workspace_tensor is not None:
            if workspace_tensor.numel() < nbytes:
                raise RuntimeError("workspace_tensor smaller than %d bytes" % nbytes)
            ws = workspace_tensor
        else:
            ws = workspace(nbytes, x.device)
        st = C.c_void_p(stream.cuda_stream) if stream is not None else stream_of(x)
        N.check(lib.ws_eval_fitness(code, ptr(population), B, L, ptr(x), V, D,
                                    ptr(constants) if K > 0 else None, K, ptr(y_target),
                                    ptr(out), ptr(out_ninvalid), C.byref(self._tmap),
                                    C.byref(opts), ptr(ws), nbytes, st))
        return out
