"""Constant fitting over the adjoint gradient, for populations of any size.

  loss_grad(...)  one launch: per-program mean squared error and its gradient with respect to the
                  constants (ws_loss_grad) -- what the reference's L-BFGS closure computes with
                  RPNBackwardFunction, [B, D] predictions and torch reductions
                  (src/warpsymbolic/gpu/optimization.py:301-311);
  lbfgs(...)      one L-BFGS per program (ws_lbfgs_adjoint) with torch.optim.LBFGS's algorithm
                  and options (strong-Wolfe line search), instead of the reference's single joint
                  L-BFGS over the sum of all programs' losses (optimization.py:281-343).

Token IDs are the 36 scalars of CudaRPNVM (vm.ids), as for the native drop-in; x is
variables-major [V, D].
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional, Sequence, Tuple

import torch

from . import _native as N
from ._tensors import check_cuda, dtype_code, ptr, stream_of, workspace


def _ids_map(ids: Sequence[int], pi_val: float, e_val: float) -> N.TokenMap:
    return N.TokenMap.from_args(*ids, pi_val=pi_val, e_val=e_val)


def _check(population, x, constants, y):
    for t, nm in ((population, "population"), (x, "x"), (constants, "constants"), (y, "y")):
        check_cuda(t, nm)
    if population.dtype != torch.uint8 or population.dim() != 2:
        raise RuntimeError("population must be uint8 [B, L]")
    if x.dim() != 2:
        raise RuntimeError("x must be [V, D] (variables-major)")
    if constants.dtype != x.dtype or y.dtype != x.dtype:
        raise RuntimeError("constants and y must have x's dtype")
    B, L = int(population.size(0)), int(population.size(1))
    V, D = int(x.size(0)), int(x.size(1))
    K = int(constants.size(1)) if constants.dim() == 2 else 0
    if constants.numel() != B * K:
        raise RuntimeError("constants must be [B, K]")
    if y.numel() != D:
        raise RuntimeError("y must have D elements")
    return B, L, V, D, K


def loss_grad(population: torch.Tensor, x: torch.Tensor, constants: torch.Tensor,
              y: torch.Tensor, ids: Sequence[int], pi_val: float = math.pi,
              e_val: float = math.e, active: Optional[torch.Tensor] = None
              ) -> Tuple[torch.Tensor, torch.Tensor]:
    """(loss [B] float64, grad [B, K] in x's dtype): loss = mean_d (pred - y)^2 per program,
    grad = d loss / d constants; infinite loss for programs without a result."""
    B, L, V, D, K = _check(population, x, constants, y)
    dev = x.device
    loss = torch.empty(B, dtype=torch.float64, device=dev)
    grad = torch.empty((B, K), dtype=x.dtype, device=dev)
    if active is not None:
        check_cuda(active, "active")
        if active.dtype != torch.int32 or active.numel() != B:
            raise RuntimeError("active must be int32 [B]")
    dt = dtype_code(x.dtype)
    lib = N.lib()
    need = C.c_size_t(0)
    N.check(lib.ws_loss_grad_workspace_bytes(dt, B, L, V, D, K, C.byref(need)))
    ws = workspace(need.value, dev)
    m = _ids_map(ids, pi_val, e_val)
    N.check(lib.ws_loss_grad(dt, ptr(population), B, L, ptr(x), V, D, ptr(constants), K, ptr(y),
                             ptr(active), ptr(loss), ptr(grad), C.byref(m), ptr(ws),
                             ws.numel(), stream_of(x)))
    return loss, grad


def lbfgs(population: torch.Tensor, x: torch.Tensor, constants: torch.Tensor, y: torch.Tensor,
          ids: Sequence[int], max_iter: int = 20, max_eval: Optional[int] = None,
          history_size: int = 10, max_ls: int = 25, lr: float = 1.0,
          tolerance_grad: float = 1e-7, tolerance_change: float = 1e-9,
          grad_clip: float = 1e4, sync_every: int = 4, pi_val: float = math.pi,
          e_val: float = math.e) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    """One torch.optim.LBFGS(line_search_fn="strong_wolfe") per program, all programs at once.

    Returns (constants after the last accepted step [B, K], their loss [B] float64, loss
    evaluations used [B] int32); `constants` itself is not modified.  max_eval defaults to
    max_iter * 5 // 4 as in torch.  grad_clip clamps every gradient before L-BFGS sees it, as the
    reference's closure does (1e4); 0 disables it."""
    B, L, V, D, K = _check(population, x, constants, y)
    if max_eval is None:
        max_eval = max_iter * 5 // 4
    dev = x.device
    out = constants.detach().clone().contiguous()
    loss = torch.empty(B, dtype=torch.float64, device=dev)
    evals = torch.zeros(B, dtype=torch.int32, device=dev)
    if B == 0:
        return out, loss, evals
    dt = dtype_code(x.dtype)
    lib = N.lib()
    need = C.c_size_t(0)
    N.check(lib.ws_lbfgs_adjoint_workspace_bytes(dt, B, L, V, D, K, int(history_size),
                                                 C.byref(need)))
    ws = workspace(need.value, dev)
    opts = N.LbfgsOpts(int(max_iter), int(max_eval), int(history_size), int(max_ls), float(lr),
                       float(tolerance_grad), float(tolerance_change), float(grad_clip),
                       int(sync_every), 0)
    m = _ids_map(ids, pi_val, e_val)
    N.check(lib.ws_lbfgs_adjoint(dt, ptr(population), B, L, ptr(x), V, D, ptr(out), K, ptr(y),
                                 C.byref(opts), ptr(loss), ptr(evals), C.byref(m), ptr(ws),
                                 ws.numel(), stream_of(x)))
    return out, loss, evals
