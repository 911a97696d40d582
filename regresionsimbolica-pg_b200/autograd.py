"""Gradient path: RPNBackwardFunction and evaluate_with_gradients, mirrors of
src/warpsymbolic/gpu/optimization.py:9-88 on top of libwarpsym.

The forward pass is the classic per-row evaluator (ws_eval_rpn, bit-identical to the
reference's eval_rpn); the backward pass is the adjoint kernel (ws_eval_rpn_backward), which
sums the per-row constant adjoints without per-row atomics.  As in the reference, the token
IDs come from a CudaRPNVM-like object and pi / e are passed as math.pi / math.e.
"""
from __future__ import annotations

import math

import torch

from . import rpn_cuda_native as _rcn

_ID_NAMES = ("PAD_ID", "id_x_start", "id_C", "id_pi", "id_e", "id_0", "id_1", "id_2", "id_3",
             "id_4", "id_5", "id_6", "id_10", "op_add", "op_sub", "op_mul", "op_div", "op_pow",
             "op_mod", "op_sin", "op_cos", "op_tan", "op_log", "op_exp", "op_sqrt", "op_abs",
             "op_neg", "op_fact", "op_floor", "op_ceil", "op_sign", "op_gamma", "op_lgamma",
             "op_asin", "op_acos", "op_atan")


def _vm_ids(vm):
    """The 36 scalar IDs in argument order, from this package's CudaRPNVM (`ids`) or from an
    object carrying them as attributes, like the reference's CudaRPNVM (cuda_vm.py:34-82)."""
    ids = getattr(vm, "ids", None)
    if ids is not None:
        return tuple(ids)
    return tuple(getattr(vm, n) for n in _ID_NAMES)


class RPNBackwardFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, population, constants, x, y_target, vm):
        B = population.shape[0]
        D = x.shape[1]
        preds = torch.empty((B, D), device=constants.device, dtype=constants.dtype)
        sp_out = torch.empty((B, D), device=constants.device, dtype=torch.int32)
        error_out = torch.zeros((B, D), device=constants.device, dtype=torch.uint8)
        x_cuda = x
        if x.ndim == 2 and x.shape[0] == D and x.shape[1] != D:
            x_cuda = x.T.contiguous()
        elif not x.is_contiguous():
            x_cuda = x.contiguous()
        ids = _vm_ids(vm)
        _rcn.eval_rpn(population.contiguous(), x_cuda, constants.contiguous(), preds, sp_out,
                      error_out, *ids, math.pi, math.e, 0)
        ctx.save_for_backward(population, constants, x_cuda)
        ctx.ids = ids
        return preds

    @staticmethod
    def backward(ctx, grad_output):
        population, constants, x_cuda = ctx.saved_tensors
        grad_constants = torch.zeros_like(constants)
        _rcn.eval_rpn_backward(population.contiguous(), x_cuda, constants.contiguous(),
                               grad_output.contiguous(), grad_constants, *ctx.ids, math.pi,
                               math.e)
        return None, grad_constants, None, None, None


def evaluate_with_gradients(population, constants, x, y_target, vm):
    """loss = sum_b mean_d (pred - y)^2 with gradients w.r.t. constants; also RMSE [B]."""
    preds = RPNBackwardFunction.apply(population, constants, x, y_target, vm)
    diff = preds - y_target.unsqueeze(0)
    mse = (diff ** 2).mean(dim=1)
    loss = mse.sum()
    return loss, torch.sqrt(mse.detach())
