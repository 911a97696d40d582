"""Drop-in for the reference extension module `rpn_cuda_native` (src/warpsymbolic/gpu/cuda/).

Same function names, argument order, keyword defaults and in-place output semantics as the
pybind11 exports (bindings.cpp:434-581); the work is done by libwarpsym.so (sm_100a kernels,
C ABI in include/warpsym.h).  Make this module importable as `rpn_cuda_native` (put this
package directory on sys.path, or see INTEGRATION.md) and the reference's
`cuda_loader.load_rpn_cuda_native()` resolves it.

Differences by design: launches go to torch's current stream (the reference uses the legacy
default stream), the GIL is released during the native call (ctypes), and indices are 64-bit.
"""
from __future__ import annotations

import ctypes as C
import importlib.util
import os
import sys

import torch


def _package():
    """The package this file belongs to, registered as `warpsymbolic_b200` (its directory name
    is not a Python identifier), also when this file is imported as top-level
    `rpn_cuda_native`."""
    name = "warpsymbolic_b200"
    if name not in sys.modules:
        here = os.path.dirname(os.path.abspath(__file__))
        spec = importlib.util.spec_from_file_location(
            name, os.path.join(here, "__init__.py"), submodule_search_locations=[here])
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


_pkg = _package()
from warpsymbolic_b200 import _native as N  # noqa: E402
from warpsymbolic_b200._tensors import check_cuda, dtype_code, ptr, stream_of, workspace  # noqa: E402


def _token_map(ids, pi_val, e_val) -> N.TokenMap:
    return N.TokenMap.from_args(*ids, pi_val=pi_val, e_val=e_val)


def eval_rpn(population, x, constants, out_preds, out_sp, out_error,
             PAD_ID, id_x_start, id_C, id_pi, id_e,
             id_0, id_1, id_2, id_3, id_4, id_5, id_6, id_10,
             op_add, op_sub, op_mul, op_div, op_pow, op_mod,
             op_sin, op_cos, op_tan, op_log, op_exp,
             op_sqrt, op_abs, op_neg,
             op_fact, op_floor, op_ceil, op_sign,
             op_gamma, op_lgamma, op_asin, op_acos, op_atan,
             pi_val, e_val, strict_mode=0):
    """Classic per-(program,row) evaluation (bindings.cpp:434 -> rpn_kernels.cu:361-429).
    Fills out_preds/out_sp/out_error ([B*D] or [B, D]) in place."""
    check_cuda(population, "population")
    check_cuda(x, "x")
    K = int(constants.size(1)) if constants.dim() > 1 else 0
    if K > 0:
        check_cuda(constants, "constants")
    B, L = int(population.size(0)), int(population.size(1))
    V, D = int(x.size(0)), int(x.size(1))
    m = _token_map((PAD_ID, id_x_start, id_C, id_pi, id_e, id_0, id_1, id_2, id_3, id_4, id_5,
                    id_6, id_10, op_add, op_sub, op_mul, op_div, op_pow, op_mod, op_sin, op_cos,
                    op_tan, op_log, op_exp, op_sqrt, op_abs, op_neg, op_fact, op_floor, op_ceil,
                    op_sign, op_gamma, op_lgamma, op_asin, op_acos, op_atan), pi_val, e_val)
    for t, nm, dt in ((out_preds, "out_preds", x.dtype), (out_sp, "out_sp", torch.int32),
                      (out_error, "out_error", torch.uint8)):
        check_cuda(t, nm)
        if t.numel() != B * D or t.dtype != dt:
            raise RuntimeError("%s must have B*D elements of dtype %s" % (nm, dt))
    N.check(N.lib().ws_eval_rpn(dtype_code(x.dtype), ptr(population), B, L, ptr(x), V, D,
                                ptr(constants) if K > 0 else None, K, ptr(out_preds),
                                ptr(out_sp), ptr(out_error), C.byref(m), int(strict_mode),
                                stream_of(x)))


def eval_rpn_fused(population, x, constants, y_target, out_rmse,
                   PAD_ID, id_x_start, id_C, id_pi, id_e,
                   id_0, id_1, id_2, id_3, id_4, id_5, id_6, id_10,
                   op_add, op_sub, op_mul, op_div, op_pow, op_mod,
                   op_sin, op_cos, op_tan, op_log, op_exp,
                   op_sqrt, op_abs, op_neg,
                   op_fact, op_floor, op_ceil, op_sign,
                   op_gamma, op_lgamma, op_asin, op_acos, op_atan,
                   pi_val, e_val, strict_mode=0, launch_mode=0):
    """Fused evaluation + RMSE (bindings.cpp:436 -> rpn_kernels.cu:2505-2594): same checks,
    envelope and error texts; out_rmse [B] written in place."""
    for t, nm in ((population, "population"), (x, "x"), (constants, "constants"),
                  (y_target, "y_target"), (out_rmse, "out_rmse")):
        check_cuda(t, nm)
    B, L = int(population.size(0)), int(population.size(1))
    V, D = int(x.size(0)), int(x.size(1))
    K = int(constants.size(1)) if constants.dim() > 1 else 0
    if population.dim() != 2:
        raise RuntimeError("population must have shape [B, L]")
    if population.dtype != torch.uint8:
        raise RuntimeError("population must use uint8 tokens")
    if x.dim() != 2:
        raise RuntimeError("x must have shape [Vars, D]")
    m = _token_map((PAD_ID, id_x_start, id_C, id_pi, id_e, id_0, id_1, id_2, id_3, id_4, id_5,
                    id_6, id_10, op_add, op_sub, op_mul, op_div, op_pow, op_mod, op_sin, op_cos,
                    op_tan, op_log, op_exp, op_sqrt, op_abs, op_neg, op_fact, op_floor, op_ceil,
                    op_sign, op_gamma, op_lgamma, op_asin, op_acos, op_atan), pi_val, e_val)
    # envelope checks first (same order as rpn_kernels.cu:2539-2545), then shapes/dtypes
    lib = N.lib()
    if not (B > 0 and L > 0):
        raise RuntimeError("population must be non-empty")
    if not (0 < V <= 4):
        raise RuntimeError("fused evaluator supports 1..4 variables")
    if L > 256:
        raise RuntimeError("fused evaluator program length exceeds 256")
    if not (0 < D <= 1024):
        raise RuntimeError("fused evaluator supports 1..1024 samples")
    if constants.dim() != 2 or int(constants.size(0)) != B:
        raise RuntimeError("constants must have shape [B, K]")
    if y_target.dim() != 1 or y_target.numel() != D:
        raise RuntimeError("y_target must have shape [D]")
    if out_rmse.dim() != 1 or out_rmse.numel() != B:
        raise RuntimeError("out_rmse must have shape [B]")
    if constants.dtype != x.dtype:
        raise RuntimeError("constants dtype must match x")
    if y_target.dtype != x.dtype:
        raise RuntimeError("y_target dtype must match x")
    if out_rmse.dtype != x.dtype:
        raise RuntimeError("out_rmse dtype must match x")
    code = dtype_code(x.dtype)
    nbytes = lib.ws_fitness_workspace_bytes(B, L, code)
    ws = workspace(nbytes, x.device)
    N.check(lib.ws_eval_rpn_fused(code, ptr(population), B, L, ptr(x), V, D,
                                  ptr(constants) if K > 0 else None, K, ptr(y_target),
                                  ptr(out_rmse), C.byref(m), int(strict_mode), int(launch_mode),
                                  ptr(ws), nbytes, stream_of(x)))
