"""Drop-in for the reference extension module `rpn_cuda_native` (src/warpsymbolic/gpu/cuda/).

Same function names, argument order, keyword defaults and in-place output semantics as the
pybind11 exports (bindings.cpp:434-581); the work is done by libwarpsym.so (sm_100a kernels,
C ABI in include/warpsym.h).  Make this module importable as `rpn_cuda_native` (put this
package directory on sys.path, or register it in sys.modules under that name before the
reference's gpu package is imported, as reference_engine.install_native does) and the
reference's `cuda_loader.load_rpn_cuda_native()` resolves it.

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


def _optional(t):
    """The reference treats an empty tensor (numel() == 0) as "not given"."""
    return None if t is None or (isinstance(t, torch.Tensor) and t.numel() == 0) else t


def _expect(t, name, dtype):
    if t.dtype != dtype:
        raise RuntimeError("%s: expected scalar type %s but found %s" % (name, dtype, t.dtype))


def validate_rpn_batch(population, token_arities, out_valid, PAD_ID):
    """Stack validity per program (bindings.cpp:462 -> rpn_kernels.cu:850-925): out_valid [B]
    (torch.bool) written in place."""
    for t, nm in ((population, "population"), (token_arities, "token_arities"),
                  (out_valid, "out_valid")):
        check_cuda(t, nm)
    _expect(population, "population", torch.uint8)
    _expect(token_arities, "token_arities", torch.int32)
    _expect(out_valid, "out_valid", torch.bool)
    B, L = int(population.size(0)), int(population.size(1))
    N.check(N.lib().ws_validate_rpn_batch(ptr(population), 1, B, L, ptr(token_arities),
                                          int(token_arities.size(0)), int(PAD_ID),
                                          N.WS_VALIDATE_KERNEL, ptr(out_valid),
                                          stream_of(population)))


def find_subtree_ranges(population, token_arities, out_starts, PAD_ID, out_lengths=None):
    """Subtree start of every position (bindings.cpp:454 -> rpn_kernels.cu:433-537):
    out_starts [B, L] int64 and, when given, out_lengths [B] int64 written in place."""
    for t, nm in ((population, "population"), (token_arities, "token_arities"),
                  (out_starts, "out_starts")):
        check_cuda(t, nm)
    out_lengths = _optional(out_lengths)
    if out_lengths is not None:
        check_cuda(out_lengths, "out_lengths")
        _expect(out_lengths, "out_lengths", torch.int64)
    _expect(population, "population", torch.uint8)
    _expect(token_arities, "token_arities", torch.int32)
    _expect(out_starts, "out_starts", torch.int64)
    B, L = int(population.size(0)), int(population.size(1))
    N.check(N.lib().ws_find_subtree_ranges(ptr(population), B, L, ptr(token_arities),
                                           int(token_arities.size(0)), int(PAD_ID),
                                           ptr(out_starts), ptr(out_lengths),
                                           stream_of(population)))


def precompute_subtree_starts(population, arities, out_starts):
    """Subtree starts by the simplifier's recurrence (bindings.cpp:506 ->
    simplify_kernels.cu:612-737): population int64 [B, L], out_starts int64 [B, L]."""
    for t, nm in ((population, "population"), (arities, "arities"), (out_starts, "out_starts")):
        check_cuda(t, nm)
    _expect(population, "population", torch.int64)
    _expect(arities, "arities", torch.int32)
    _expect(out_starts, "out_starts", torch.int64)
    B, L = int(population.size(0)), int(population.size(1))
    N.check(N.lib().ws_precompute_subtree_starts(ptr(population), B, L, ptr(arities),
                                                 int(arities.size(0)), ptr(out_starts),
                                                 stream_of(population)))


def tournament_selection(fitness, errors, rand_idx, rand_cases, selected_idx, lengths,
                         mad_eps=None):
    """Tournament winners (bindings.cpp:468 -> rpn_kernels.cu:1535-1715): selected_idx [B] int64
    written in place.  errors / rand_cases / lengths / mad_eps may be empty tensors."""
    for t, nm in ((fitness, "fitness"), (rand_idx, "rand_idx"), (selected_idx, "selected_idx")):
        check_cuda(t, nm)
    errors, rand_cases = _optional(errors), _optional(rand_cases)
    lengths, mad_eps = _optional(lengths), _optional(mad_eps)
    for t, nm, dt in ((errors, "errors", torch.float32), (rand_cases, "rand_cases", torch.int32),
                      (lengths, "lengths", torch.float32), (mad_eps, "mad_eps", torch.float32)):
        if t is not None:
            check_cuda(t, nm)
            _expect(t, nm, dt)
    _expect(fitness, "fitness", torch.float32)
    _expect(rand_idx, "rand_idx", torch.int64)
    _expect(selected_idx, "selected_idx", torch.int64)
    B = int(fitness.size(0))
    T = int(rand_idx.size(1))
    n_data = int(errors.size(1)) if errors is not None else 0
    N.check(N.lib().ws_tournament_select(ptr(fitness), B, ptr(errors), n_data, ptr(rand_idx), T,
                                         ptr(rand_cases), ptr(lengths), ptr(mad_eps),
                                         ptr(selected_idx), stream_of(fitness)))


def eval_rpn_backward(population, x, constants, grad_output, grad_constants,
                      PAD_ID, id_x_start, id_C, id_pi, id_e,
                      id_0, id_1, id_2, id_3, id_4, id_5, id_6, id_10,
                      op_add, op_sub, op_mul, op_div, op_pow, op_mod,
                      op_sin, op_cos, op_tan, op_log, op_exp,
                      op_sqrt, op_abs, op_neg,
                      op_fact, op_floor, op_ceil, op_sign,
                      op_gamma, op_lgamma, op_asin, op_acos, op_atan,
                      pi_val, e_val):
    """Adjoint of the program outputs w.r.t. the constants (bindings.cpp:511 ->
    backward_kernels.cu:13-335): grad_constants [B, K] += sum_d grad_output[b, d] * dpred/dC."""
    for t, nm in ((population, "population"), (x, "x"), (constants, "constants"),
                  (grad_output, "grad_output"), (grad_constants, "grad_constants")):
        check_cuda(t, nm)
    _expect(population, "population", torch.uint8)
    B, L = int(population.size(0)), int(population.size(1))
    V, D = int(x.size(0)), int(x.size(1))
    K = int(constants.size(1)) if constants.dim() > 1 else 0
    for t, nm in ((constants, "constants"), (grad_output, "grad_output"),
                  (grad_constants, "grad_constants")):
        _expect(t, nm, x.dtype)
    if grad_output.numel() != B * D:
        raise RuntimeError("grad_output must have B*D elements")
    if grad_constants.numel() != B * K:
        raise RuntimeError("grad_constants must have B*K elements")
    m = _token_map((PAD_ID, id_x_start, id_C, id_pi, id_e, id_0, id_1, id_2, id_3, id_4, id_5,
                    id_6, id_10, op_add, op_sub, op_mul, op_div, op_pow, op_mod, op_sin, op_cos,
                    op_tan, op_log, op_exp, op_sqrt, op_abs, op_neg, op_fact, op_floor, op_ceil,
                    op_sign, op_gamma, op_lgamma, op_asin, op_acos, op_atan), pi_val, e_val)
    # scratch for grouping the programs by tape size (torch's allocator, stream-ordered)
    need = C.c_size_t(0)
    N.check(N.lib().ws_eval_rpn_backward_workspace_bytes(B, C.byref(need)))
    ws = workspace(need.value, x.device)
    N.check(N.lib().ws_eval_rpn_backward_ws(dtype_code(x.dtype), ptr(population), B, L, ptr(x), V,
                                            D, ptr(constants), K, ptr(grad_output),
                                            ptr(grad_constants), C.byref(m), ptr(ws), ws.numel(),
                                            stream_of(x)))


def decode_rpn(population, constants, vocab, arities, PAD_ID, precision=4):
    """RPN -> infix strings (bindings.cpp:450 -> decoder.cpp:32-152), on the host like the
    reference: population uint8 [B, L], constants float32/float64 [B, K] on any device."""
    import numpy as np
    pop = population.detach().cpu()
    if pop.dtype != torch.uint8:
        raise RuntimeError("population: expected scalar type Byte but found %s" % pop.dtype)
    pop = pop.contiguous()
    cst = constants.detach().cpu().contiguous()
    if cst.dtype not in (torch.float32, torch.float64):
        raise RuntimeError("constants: expected scalar type Double but found %s" % cst.dtype)
    B, L = int(pop.size(0)), int(pop.size(1))
    K = int(cst.size(1))
    voc = (C.c_char_p * max(len(vocab), 1))(*[str(v).encode("utf-8") for v in vocab])
    ar = np.ascontiguousarray(np.asarray(list(arities), dtype=np.int64).astype(np.int32))
    offsets = np.zeros(B + 1, dtype=np.int64)
    need = C.c_size_t(0)
    lib = N.lib()
    args = (C.c_void_p(pop.data_ptr()), B, L, C.c_void_p(cst.data_ptr()),
            N.WS_F32 if cst.dtype == torch.float32 else N.WS_F64, K, voc, len(vocab),
            C.c_void_p(ar.ctypes.data), ar.size, int(PAD_ID), int(precision))
    st = lib.ws_decode_rpn(*args, None, 0, C.c_void_p(offsets.ctypes.data), C.byref(need))
    if st not in (N.WS_OK, 3):
        N.check(st)
    buf = C.create_string_buffer(max(int(need.value), 1))
    N.check(lib.ws_decode_rpn(*args, buf, int(need.value), C.c_void_p(offsets.ctypes.data),
                              C.byref(need)))
    raw = buf.raw
    return [raw[offsets[i]:offsets[i + 1] - 1].decode("utf-8") for i in range(B)]


def pso_update(pos, vel, pbest, gbest, r1, r2, w, c1, c2):
    """PSO velocity / position step (bindings.cpp:470 -> pso_kernels.cu:29-187), in place on
    pos and vel [B, P, K]."""
    check_cuda(pos, "pos")
    check_cuda(vel, "vel")
    B, P, K = (int(v) for v in pos.shape)
    for t, nm in ((vel, "vel"), (pbest, "pbest"), (gbest, "gbest"), (r1, "r1"), (r2, "r2")):
        check_cuda(t, nm)
        _expect(t, nm, pos.dtype)
    N.check(N.lib().ws_pso_update(dtype_code(pos.dtype), ptr(pos), ptr(vel), ptr(pbest),
                                  ptr(gbest), ptr(r1), ptr(r2), float(w), float(c1), float(c2),
                                  B, P, K, stream_of(pos)))


def pso_update_bests(current_err, pbest_err, pbest_pos, current_pos, gbest_err, gbest_pos):
    """Personal / swarm bests (bindings.cpp:471 -> pso_kernels.cu:74-233), in place."""
    for t, nm in ((current_err, "current_err"), (pbest_err, "pbest_err"),
                  (pbest_pos, "pbest_pos"), (current_pos, "current_pos"),
                  (gbest_err, "gbest_err"), (gbest_pos, "gbest_pos")):
        check_cuda(t, nm)
        _expect(t, nm, pbest_err.dtype)
    B, P = int(pbest_err.size(0)), int(pbest_err.size(1))
    K = int(pbest_pos.size(2))
    N.check(N.lib().ws_pso_update_bests(dtype_code(pbest_err.dtype), ptr(current_err),
                                        ptr(pbest_err), ptr(pbest_pos), ptr(current_pos),
                                        ptr(gbest_err), ptr(gbest_pos), B, P, K,
                                        stream_of(pbest_err)))


def fused_pso(population, init_consts, x, y_target, out_gbest_pos, out_gbest_err,
              num_particles, num_steps, w, c1, c2, const_min, const_max,
              PAD_ID, id_x_start, id_C, id_pi, id_e,
              id_0, id_1, id_2, id_3, id_4, id_5, id_6, id_10,
              op_add, op_sub, op_mul, op_div, op_pow, op_mod,
              op_sin, op_cos, op_tan, op_log, op_exp,
              op_sqrt, op_abs, op_neg,
              op_fact, op_floor, op_ceil, op_sign,
              op_gamma, op_lgamma, op_asin, op_acos, op_atan,
              pi_val, e_val, rng_seed):
    """The whole PSO loop in one launch (bindings.cpp:510 -> fused_pso_kernels.cu:208-515):
    writes out_gbest_pos [B, K] and out_gbest_err [B]."""
    for t, nm in ((population, "population"), (init_consts, "init_consts"), (x, "x"),
                  (y_target, "y_target")):
        check_cuda(t, nm)
    B, L = int(population.size(0)), int(population.size(1))
    K = int(init_consts.size(1))
    V, D = int(x.size(0)), int(x.size(1))
    m = _token_map((PAD_ID, id_x_start, id_C, id_pi, id_e, id_0, id_1, id_2, id_3, id_4, id_5,
                    id_6, id_10, op_add, op_sub, op_mul, op_div, op_pow, op_mod, op_sin, op_cos,
                    op_tan, op_log, op_exp, op_sqrt, op_abs, op_neg, op_fact, op_floor, op_ceil,
                    op_sign, op_gamma, op_lgamma, op_asin, op_acos, op_atan), pi_val, e_val)
    lib = N.lib()
    if x.dtype == torch.float32:
        for t, nm in ((init_consts, "init_consts"), (y_target, "y_target"),
                      (out_gbest_pos, "out_gbest_pos"), (out_gbest_err, "out_gbest_err")):
            if t.dtype != x.dtype:
                raise RuntimeError("%s dtype must match x" % nm)
    code = N.WS_F32 if x.dtype == torch.float32 else N.WS_F64
    N.check(lib.ws_fused_pso(code, ptr(population), B, L, ptr(init_consts), K, ptr(x), V, D,
                             ptr(y_target), ptr(out_gbest_pos), ptr(out_gbest_err),
                             int(num_particles), int(num_steps), float(w), float(c1), float(c2),
                             float(const_min), float(const_max), C.byref(m),
                             int(rng_seed) & 0xFFFFFFFFFFFFFFFF, stream_of(x)))


def lbfgs_optimize(population, constants, x, y_target, out_rmse, max_iter=20, history_size=10,
                   gtol=1e-7, const_min=-25.0, const_max=25.0, PAD_ID=None, id_x_start=None,
                   id_C=None, id_pi=None, id_e=None, id_0=None, id_1=None, id_2=None, id_3=None,
                   id_4=None, id_5=None, id_6=None, id_10=None, op_add=None, op_sub=None,
                   op_mul=None, op_div=None, op_pow=None, op_mod=None, op_sin=None, op_cos=None,
                   op_tan=None, op_log=None, op_exp=None, op_sqrt=None, op_abs=None,
                   op_neg=None, op_fact=None, op_floor=None, op_ceil=None, op_sign=None,
                   op_gamma=None, op_lgamma=None, op_asin=None, op_acos=None, op_atan=None,
                   pi_val=None, e_val=None):
    """Constant fitting with the reference's L-BFGS kernel (bindings.cpp:542-563 ->
    lbfgs_kernels.cu:214-694): constants [B, K] updated in place, out_rmse [B] written."""
    ids = (PAD_ID, id_x_start, id_C, id_pi, id_e, id_0, id_1, id_2, id_3, id_4, id_5, id_6,
           id_10, op_add, op_sub, op_mul, op_div, op_pow, op_mod, op_sin, op_cos, op_tan,
           op_log, op_exp, op_sqrt, op_abs, op_neg, op_fact, op_floor, op_ceil, op_sign,
           op_gamma, op_lgamma, op_asin, op_acos, op_atan)
    if any(v is None for v in ids) or pi_val is None or e_val is None:
        raise TypeError("lbfgs_optimize: the token IDs, pi_val and e_val are required")
    for t, nm in ((population, "population"), (constants, "constants"), (x, "x"),
                  (y_target, "y_target"), (out_rmse, "out_rmse")):
        check_cuda(t, nm)
    B, L = int(population.size(0)), int(population.size(1))
    K = int(constants.size(1))
    V, D = int(x.size(0)), int(x.size(1))
    m = _token_map(ids, pi_val, e_val)
    N.check(N.lib().ws_lbfgs_optimize(dtype_code(x.dtype), ptr(population), B, L, ptr(constants),
                                      K, ptr(x), V, D, ptr(y_target), ptr(out_rmse),
                                      int(max_iter), int(history_size), float(gtol),
                                      float(const_min), float(const_max), C.byref(m),
                                      stream_of(x)))


def simplify_batch(population, arities, val_table, literal_ids, literal_vals, max_passes,
                   op_plus, op_minus, op_mult, op_div, op_neg, op_mod, op_pow,
                   op_sin, op_cos, op_tan, op_asin, op_acos, op_atan,
                   op_log, op_exp, op_sqrt, op_abs, op_gamma, op_lgamma,
                   op_floor, op_ceil, op_sign,
                   id_0, id_1, id_2, id_3, id_4, id_5, id_6):
    """Rule-based simplification in place (bindings.cpp:505 -> simplify_kernels.cu:100-713):
    population int64 [B, L] is rewritten."""
    for t, nm in ((population, "population"), (arities, "arities"), (val_table, "val_table"),
                  (literal_ids, "literal_ids"), (literal_vals, "literal_vals")):
        check_cuda(t, nm)
    _expect(population, "population", torch.int64)
    _expect(arities, "arities", torch.int32)
    _expect(val_table, "val_table", torch.float32)
    _expect(literal_ids, "literal_ids", torch.int64)
    _expect(literal_vals, "literal_vals", torch.float32)
    ids = N.SimplifyIds(*[int(v) for v in (
        op_plus, op_minus, op_mult, op_div, op_neg, op_mod, op_pow, op_sin, op_cos, op_tan,
        op_asin, op_acos, op_atan, op_log, op_exp, op_sqrt, op_abs, op_gamma, op_lgamma,
        op_floor, op_ceil, op_sign, id_0, id_1, id_2, id_3, id_4, id_5, id_6)])
    B, L = int(population.size(0)), int(population.size(1))
    N.check(N.lib().ws_simplify_batch(ptr(population), B, L, ptr(arities), int(arities.size(0)),
                                      ptr(val_table), ptr(literal_ids), ptr(literal_vals),
                                      int(literal_ids.size(0)), int(max_passes), C.byref(ids),
                                      stream_of(population)))


# ---- genetic operators and best tracking (next-tier exports of bindings.cpp) -----------------
def _u8_ptr_n(t, name):
    check_cuda(t, name)
    _expect(t, name, torch.uint8)
    return ptr(t) if t.numel() > 0 else None, int(t.numel())


def mutate_population(population, rand_floats, rand_ints, token_arities, arity_0_ids,
                      arity_1_ids, arity_2_ids, mutation_rate, PAD_ID):
    """Point mutation from pre-drawn randoms, in place (bindings.cpp:457 ->
    rpn_kernels.cu:772-845)."""
    for t, nm in ((population, "population"), (rand_floats, "rand_floats"),
                  (rand_ints, "rand_ints"), (token_arities, "token_arities")):
        check_cuda(t, nm)
    _expect(population, "population", torch.uint8)
    _expect(rand_floats, "rand_floats", torch.float32)
    _expect(rand_ints, "rand_ints", torch.int64)
    _expect(token_arities, "token_arities", torch.int32)
    B, L = int(population.size(0)), int(population.size(1))
    if rand_floats.numel() < B * L or rand_ints.numel() < B * L:
        raise RuntimeError("rand_floats and rand_ints must hold [B, L] values")
    a0, n0 = _u8_ptr_n(arity_0_ids, "arity_0_ids")
    a1, n1 = _u8_ptr_n(arity_1_ids, "arity_1_ids")
    a2, n2 = _u8_ptr_n(arity_2_ids, "arity_2_ids")
    N.check(N.lib().ws_mutate_population(ptr(population), B, L, ptr(rand_floats), ptr(rand_ints),
                                         ptr(token_arities), int(token_arities.size(0)), a0, n0,
                                         a1, n1, a2, n2, float(mutation_rate), int(PAD_ID),
                                         stream_of(population)))


def crossover_splicing(parent1, parent2, starts1, ends1, starts2, ends2, child1, child2, PAD_ID,
                       cx_mask=None):
    """Subtree splicing of parent pairs into children (bindings.cpp:458 ->
    rpn_kernels.cu:927-1016,1266-1300)."""
    for t, nm in ((parent1, "parent1"), (parent2, "parent2"), (child1, "child1"),
                  (child2, "child2")):
        check_cuda(t, nm)
        _expect(t, nm, torch.uint8)
    for t, nm in ((starts1, "starts1"), (ends1, "ends1"), (starts2, "starts2"), (ends2, "ends2")):
        check_cuda(t, nm)
        _expect(t, nm, torch.int64)
    N_, L = int(parent1.size(0)), int(parent1.size(1))
    mask = _optional(cx_mask)
    if mask is not None:
        check_cuda(mask, "cx_mask")
        _expect(mask, "cx_mask", torch.bool)
    N.check(N.lib().ws_crossover_splicing(ptr(parent1), ptr(parent2), N_, L, ptr(starts1),
                                          ptr(ends1), ptr(starts2), ptr(ends2), ptr(child1),
                                          ptr(child2), int(PAD_ID), ptr(mask),
                                          stream_of(parent1)))


def constant_perturbation(constants, rate, sigma, c_min, c_max, seed):
    """In-place multiplicative constant noise (bindings.cpp:463 -> rpn_kernels.cu:1455-1535)."""
    check_cuda(constants, "constants")
    if constants.numel() == 0 or rate <= 0.0 or sigma <= 0.0:
        return
    B, K = int(constants.size(0)), int(constants.size(1))
    N.check(N.lib().ws_constant_perturbation(dtype_code(constants.dtype), ptr(constants), B, K,
                                             float(rate), float(sigma), float(c_min),
                                             float(c_max), int(seed) & 0xFFFFFFFF,
                                             stream_of(constants)))


def generate_random_rpn(population, terminal_ids, unary_ids, binary_ids, seed, term_weight,
                        unary_weight, bin_weight):
    """Valid random programs, one per row (bindings.cpp:507 -> genrand_kernels.cu:70-210)."""
    check_cuda(population, "population")
    _expect(population, "population", torch.uint8)
    t, nt = _u8_ptr_n(terminal_ids, "terminal_ids")
    if nt <= 0:
        raise RuntimeError("Must have at least one terminal token")
    u, nu = _u8_ptr_n(unary_ids, "unary_ids")
    b, nb = _u8_ptr_n(binary_ids, "binary_ids")
    B, L = int(population.size(0)), int(population.size(1))
    N.check(N.lib().ws_generate_random_rpn(ptr(population), B, L, t, nt, u, nu, b, nb,
                                           int(seed) & 0xFFFFFFFFFFFFFFFF, float(term_weight),
                                           float(unary_weight), float(bin_weight),
                                           stream_of(population)))


def update_best(population, constants, fitness, tracker_rpn, tracker_consts, tracker_rmse,
                tracker_idx, tracker_gen, tracker_len, tracker_updated, current_generation,
                tolerance=1e-9):
    """Device-side best tracker (bindings.cpp:565 -> best_tracker_kernels.cu:47-136,238-282);
    one block reduces every program (see include/warpsym.h on the reference's block race)."""
    for t, nm in ((population, "population"), (constants, "constants"), (fitness, "fitness")):
        check_cuda(t, nm)
    _expect(population, "population", torch.int64)
    _expect(constants, "constants", torch.float32)
    _expect(fitness, "fitness", torch.float32)
    B, L = int(population.size(0)), int(population.size(1))
    K = int(constants.size(1))
    N.check(N.lib().ws_update_best(ptr(population), B, L, ptr(constants), K, ptr(fitness),
                                   ptr(tracker_rpn), ptr(tracker_consts), ptr(tracker_rmse),
                                   ptr(tracker_idx), ptr(tracker_gen), ptr(tracker_len),
                                   ptr(tracker_updated), int(current_generation), float(tolerance),
                                   stream_of(fitness)))


def check_improvement(fitness, tracked_rmse, improved, tolerance=1e-9):
    """improved[0] = min(fitness) < tracked_rmse[0] - tolerance, without a host sync
    (bindings.cpp:572 -> best_tracker_kernels.cu:141-173,284-305)."""
    check_cuda(fitness, "fitness")
    _expect(fitness, "fitness", torch.float32)
    N.check(N.lib().ws_check_improvement(ptr(fitness), int(fitness.size(0)), ptr(tracked_rmse),
                                         ptr(improved), float(tolerance), stream_of(fitness)))


def batch_update_best(population, constants, fitness, best_rpn, best_consts, best_rmse, best_idx,
                      tolerance=1e-9):
    """Single-block best update used by the generation loop (bindings.cpp:576 ->
    best_tracker_kernels.cu:178-231,307-340)."""
    for t, nm in ((population, "population"), (constants, "constants"), (fitness, "fitness")):
        check_cuda(t, nm)
    _expect(population, "population", torch.uint8)
    _expect(constants, "constants", torch.float32)
    _expect(fitness, "fitness", torch.float32)
    B, L = int(population.size(0)), int(population.size(1))
    K = int(constants.size(1))
    N.check(N.lib().ws_batch_update_best(ptr(population), B, L, ptr(constants), K, ptr(fitness),
                                         ptr(best_rpn), ptr(best_consts), ptr(best_rmse),
                                         ptr(best_idx), float(tolerance), stream_of(fitness)))


# ---- structural hashing and deduplication (diversity exports of bindings.cpp) ----------------
def compute_population_hashes(population, hashes, var_presence, PAD_ID, id_x_start, num_vars):
    """Polynomial hashes [B] int64 and, when var_presence is non-empty, used-variable masks
    [B] int32 (bindings.cpp:513 -> diversity_kernels.cu:29-108)."""
    check_cuda(population, "population")
    check_cuda(hashes, "hashes")
    _expect(population, "population", torch.uint8)
    _expect(hashes, "hashes", torch.int64)
    vp = _optional(var_presence)
    if vp is not None:
        check_cuda(vp, "var_presence")
        _expect(vp, "var_presence", torch.int32)
    B, L = int(population.size(0)), int(population.size(1))
    N.check(N.lib().ws_population_hashes(ptr(population), B, L, ptr(hashes), ptr(vp), int(PAD_ID),
                                         int(id_x_start), int(num_vars), stream_of(population)))


def compute_var_presence(population, var_presence, PAD_ID, id_x_start, num_vars):
    """Used-variable bitmask per program (bindings.cpp:536 -> diversity_kernels.cu:465-515)."""
    check_cuda(population, "population")
    check_cuda(var_presence, "var_presence")
    _expect(population, "population", torch.uint8)
    _expect(var_presence, "var_presence", torch.int32)
    B, L = int(population.size(0)), int(population.size(1))
    N.check(N.lib().ws_population_hashes(ptr(population), B, L, None, ptr(var_presence),
                                         int(PAD_ID), int(id_x_start), int(num_vars),
                                         stream_of(population)))


def structural_dedup(hashes, hash_table, duplicate_mask, original_index):
    """Duplicate flags and originals by hash (bindings.cpp:518 -> diversity_kernels.cu:121-238);
    hash_table [2^20] int64 filled with -1 by the caller.  A group's original is its lowest
    index."""
    for t, nm, dt in ((hashes, "hashes", torch.int64), (hash_table, "hash_table", torch.int64),
                      (duplicate_mask, "duplicate_mask", torch.int32),
                      (original_index, "original_index", torch.int64)):
        check_cuda(t, nm)
        _expect(t, nm, dt)
    if hash_table.numel() < int(N.lib().ws_dedup_table_slots()):
        raise RuntimeError("hash_table must hold %d entries" % N.lib().ws_dedup_table_slots())
    N.check(N.lib().ws_structural_dedup(ptr(hashes), int(hashes.size(0)), ptr(hash_table),
                                        ptr(duplicate_mask), ptr(original_index),
                                        stream_of(hashes)))


def count_unique(duplicate_mask):
    """Number of programs whose duplicate flag is 0 (bindings.cpp:522 ->
    diversity_kernels.cu:362-405); a host integer, as the reference returns."""
    check_cuda(duplicate_mask, "duplicate_mask")
    _expect(duplicate_mask, "duplicate_mask", torch.int32)
    out = torch.zeros(1, dtype=torch.int64, device=duplicate_mask.device)
    N.check(N.lib().ws_count_unique(ptr(duplicate_mask), int(duplicate_mask.size(0)), ptr(out),
                                    stream_of(duplicate_mask)))
    return int(out.item())


def get_replacement_positions(duplicate_mask, replacement_positions, n_replacements):
    """Indices of the duplicates, ascending, and their number (bindings.cpp:526 ->
    diversity_kernels.cu:410-460); returns the number as a host integer."""
    for t, nm, dt in ((duplicate_mask, "duplicate_mask", torch.int32),
                      (replacement_positions, "replacement_positions", torch.int64),
                      (n_replacements, "n_replacements", torch.int64)):
        check_cuda(t, nm)
        _expect(t, nm, dt)
    n_replacements.zero_()
    N.check(N.lib().ws_replacement_positions(ptr(duplicate_mask), int(duplicate_mask.size(0)),
                                             ptr(replacement_positions), ptr(n_replacements),
                                             stream_of(duplicate_mask)))
    return int(n_replacements.item())


def fitness_sharing_penalty(population, n_islands, island_size, threshold, hash_len=8):
    """Per-island sharing penalty [B] float32 (bindings.cpp:530 -> diversity_kernels.cu:224-355)."""
    check_cuda(population, "population")
    _expect(population, "population", torch.uint8)
    B, L = int(population.size(0)), int(population.size(1))
    slots = int(N.lib().ws_sharing_table_slots())
    dev = population.device
    keys = torch.full((int(n_islands), slots), -1, dtype=torch.int64, device=dev)
    counts = torch.zeros((int(n_islands), slots), dtype=torch.int32, device=dev)
    out = torch.empty(B, dtype=torch.float32, device=dev)
    N.check(N.lib().ws_fitness_sharing_penalty(ptr(population), B, L, int(n_islands),
                                               int(island_size), int(threshold), int(hash_len),
                                               ptr(keys), ptr(counts), ptr(out),
                                               stream_of(population)))
    return out


def _f32(v) -> float:
    """A Python number as the float32 the reference's pybind `float` parameters receive."""
    import numpy as np
    return float(np.float32(v))


def evolve_generation(population, constants, fitness, abs_errors, X, Y_target, lengths,
                      token_arities, arity_0_ids, arity_1_ids, arity_2_ids, mutation_bank,
                      mad_eps, mutation_rate, crossover_rate, tournament_size, pso_steps,
                      pso_particles, pso_w, pso_c1, pso_c2, PAD_ID,
                      id_x_start, id_C, id_pi, id_e,
                      id_0, id_1, id_2, id_3, id_4, id_5, id_6, id_10,
                      op_add, op_sub, op_mul, op_div, op_pow, op_mod,
                      op_sin, op_cos, op_tan, op_log, op_exp,
                      op_sqrt, op_abs, op_neg,
                      op_fact, op_floor, op_ceil, op_sign,
                      op_gamma, op_lgamma, op_asin, op_acos, op_atan,
                      pi_val, e_val, n_islands=1, cached_p1_src=None, cached_p2_src=None,
                      cached_copy_src=None, cached_island_base=None, rng_seed=0, generation=0):
    """One generation (bindings.cpp:474 -> rpn_kernels.cu:1810-2237): island tournament with
    elitism at index 0, subtree crossover of fixed parent pairs with fused point mutation, copies
    for the unpaired, SBX of constants and their transfer along the spliced `C` tokens,
    structural (bank) and hoist mutation, then `pso_steps` PSO steps over `pso_particles`
    particles.  Returns [population, constants, fitness] (fitness empty without PSO).

    The random draws are torch's, on the current CUDA generator, with the reference's shapes and
    order, and every device step gives the reference kernel's bytes / floats, so the same seed
    gives the same generation.  `cached_island_base` is accepted and unused, as in the
    reference."""
    from warpsymbolic_b200._native import PointMutation
    for t, nm in ((population, "population"), (constants, "constants"), (fitness, "fitness"),
                  (X, "X"), (Y_target, "Y_target"), (token_arities, "token_arities")):
        check_cuda(t, nm)
    _expect(population, "population", torch.uint8)
    _expect(constants, "constants", torch.float32)
    _expect(token_arities, "token_arities", torch.int32)
    for t, nm in ((arity_0_ids, "arity_0_ids"), (arity_1_ids, "arity_1_ids"),
                  (arity_2_ids, "arity_2_ids")):
        if t.numel() > 0:
            check_cuda(t, nm)
            _expect(t, nm, torch.uint8)
    dev = population.device
    B, L = int(population.size(0)), int(population.size(1))
    K = int(constants.size(1))
    n_data = int(X.size(1))
    T = int(tournament_size)
    vocab = int(token_arities.numel())
    lib = N.lib()
    st = stream_of(population)
    i32 = dict(dtype=torch.int32, device=dev)
    i64 = dict(dtype=torch.int64, device=dev)
    f32 = dict(dtype=torch.float32, device=dev)
    mutation_rate, crossover_rate = _f32(mutation_rate), _f32(crossover_rate)

    # 1. selection
    sel_size = max(1, B // n_islands) if n_islands > 1 else B
    rand_offsets = torch.randint(0, sel_size, (B, T), **i32)
    winner = torch.empty(B, **i64)
    has_err = abs_errors is not None and abs_errors.numel() > 0
    rand_cases = torch.randint(0, n_data, (B,), **i32) if has_err else torch.empty(0, **i32)
    fit32 = fitness if fitness.dtype == torch.float32 else fitness.to(torch.float32)
    err32 = (abs_errors if abs_errors.dtype == torch.float32 else abs_errors.to(torch.float32)) \
        if has_err else None
    len32 = lengths if (lengths is None or lengths.numel() == 0
                        or lengths.dtype == torch.float32) else lengths.to(torch.float32)
    mad32 = mad_eps if (mad_eps is None or mad_eps.numel() == 0
                        or mad_eps.dtype == torch.float32) else mad_eps.to(torch.float32)
    fit32, rand_offsets = fit32.contiguous(), rand_offsets.contiguous()
    err32 = err32.contiguous() if err32 is not None else None
    len32 = _optional(len32.contiguous()) if len32 is not None else None
    mad32 = _optional(mad32.contiguous()) if mad32 is not None else None
    N.check(lib.ws_tournament_select_offsets(ptr(fit32), B, ptr(err32),
                                             n_data if has_err else 0, ptr(rand_offsets), T,
                                             ptr(rand_cases if has_err else None), ptr(len32),
                                             ptr(mad32), sel_size, int(n_islands), ptr(winner),
                                             st))
    winner[0] = torch.argmin(fit32)

    # 2. crossover pairs inside islands (slot 0 holds the elite)
    island_size = B // n_islands
    if (cached_p1_src is not None and cached_p2_src is not None and cached_copy_src is not None
            and cached_p1_src.numel() == cached_p2_src.numel() and cached_copy_src.numel() > 0):
        p1_src, p2_src, copy_src = cached_p1_src, cached_p2_src, cached_copy_src
    else:
        p1_parts, p2_parts, copy_parts = [], [], [torch.zeros(1, **i64)]
        for k in range(n_islands):
            start, end = k * island_size, (k + 1) * island_size
            avail_start = start + 1 if k == 0 else start
            avail_len = end - avail_start
            pairs = int(avail_len / 2)  # C++ integer division
            if pairs > 0:
                p1 = torch.arange(avail_start, avail_start + 2 * pairs, 2, **i64)
                p1_parts.append(p1)
                p2_parts.append(p1 + 1)
            if avail_len % 2 != 0:
                copy_parts.append(torch.full((1,), end - 1, **i64))
        p1_src = torch.cat(p1_parts).contiguous() if p1_parts else torch.empty(0, **i64)
        p2_src = torch.cat(p2_parts).contiguous() if p2_parts else torch.empty(0, **i64)
        copy_src = torch.cat(copy_parts).contiguous()
    n_pairs = int(p1_src.size(0))
    p1_w = winner.index_select(0, p1_src)
    p2_w = winner.index_select(0, p2_src)
    copy_w = winner.index_select(0, copy_src)
    cx_prob = torch.rand(n_pairs, **f32)
    cx_candidate = cx_prob < crossover_rate
    len1, len2 = torch.empty(n_pairs, **i64), torch.empty(n_pairs, **i64)
    rand_e1 = torch.rand(n_pairs, **f32)
    rand_e2 = torch.rand(n_pairs, **f32)
    s1, e1 = torch.empty(n_pairs, **i64), torch.empty(n_pairs, **i64)
    s2, e2 = torch.empty(n_pairs, **i64), torch.empty(n_pairs, **i64)
    N.check(lib.ws_subtree_pick(ptr(population), ptr(p1_w), n_pairs, L, ptr(token_arities),
                                vocab, ptr(rand_e1), ptr(len1), ptr(s1), ptr(e1), int(PAD_ID), st))
    N.check(lib.ws_subtree_pick(ptr(population), ptr(p2_w), n_pairs, L, ptr(token_arities),
                                vocab, ptr(rand_e2), ptr(len2), ptr(s2), ptr(e2), int(PAD_ID), st))
    cx_mask = torch.empty(n_pairs, dtype=torch.bool, device=dev)
    N.check(lib.ws_splice_valid(ptr(len1), ptr(len2), ptr(s1), ptr(e1), ptr(s2), ptr(e2),
                                ptr(cx_candidate), ptr(cx_mask), n_pairs, L, st))
    u_sbx = torch.rand(n_pairs, K, **f32)
    mask_sbx = torch.rand(n_pairs, K, **f32)
    mut_rand = torch.rand(B, **f32)
    has_bank = mutation_bank is not None and mutation_bank.numel() > 0
    point_cut = _f32(0.5 if has_bank else 0.8)
    mut = PointMutation(ptr(token_arities).value, vocab, int(arity_0_ids.numel()),
                        int(arity_1_ids.numel()), int(arity_2_ids.numel()),
                        ptr(arity_0_ids).value, ptr(arity_1_ids).value, ptr(arity_2_ids).value,
                        mutation_rate, 0, int(rng_seed) & 0xFFFFFFFFFFFFFFFF,
                        int(generation) & 0xFFFFFFFFFFFFFFFF)
    offspring = torch.empty_like(population)
    N.check(lib.ws_splice_rows(ptr(population), ptr(population), ptr(p1_w), ptr(p2_w),
                               ptr(p1_src), ptr(p2_src), ptr(s1), ptr(e1), ptr(s2), ptr(e2),
                               ptr(cx_mask), ptr(offspring), ptr(offspring), n_pairs, L,
                               int(PAD_ID), ptr(mut_rand), point_cut, C.byref(mut), st))
    offspring.index_copy_(0, copy_src, population.index_select(0, copy_w))
    N.check(lib.ws_mutate_rows(ptr(offspring), ptr(copy_src), int(copy_src.numel()), L,
                               ptr(mut_rand), point_cut, C.byref(mut), int(PAD_ID), st))
    consts1 = torch.empty(n_pairs, K, **f32)
    consts2 = torch.empty(n_pairs, K, **f32)
    N.check(lib.ws_sbx_constants(ptr(constants), ptr(p1_w), ptr(p2_w), ptr(u_sbx), ptr(mask_sbx),
                                 ptr(consts1), ptr(consts2), n_pairs, K, 2.0, st))
    offspring_consts = torch.empty_like(constants)
    N.check(lib.ws_splice_constants(ptr(population), ptr(p1_w), ptr(p2_w), ptr(consts1),
                                    ptr(consts2), ptr(s1), ptr(e1), ptr(s2), ptr(e2),
                                    ptr(cx_mask), ptr(offspring_consts), ptr(p1_src),
                                    ptr(p2_src), n_pairs, L, K, int(id_C), st))
    offspring_consts.index_copy_(0, copy_src, constants.index_select(0, copy_w))

    # 3. structural and hoist mutation (never the elite)
    import numpy as np
    mr = np.float32(mutation_rate)
    hoist_cut = float(np.float32(0.8) + np.float32(0.2) * mr)
    hoist_mask = (mut_rand >= 0.8) & (mut_rand < hoist_cut)
    if has_bank:
        struct_cut = float(np.float32(0.5) + np.float32(0.3) * mr)
        struct_mask = (mut_rand >= 0.5) & (mut_rand < struct_cut)
        struct_mask[0] = False
    hoist_mask[0] = False
    if has_bank:
        check_cuda(mutation_bank, "mutation_bank")
        _expect(mutation_bank, "mutation_bank", torch.uint8)
        struct_idx = torch.nonzero(struct_mask).squeeze(1)
        n_struct = int(struct_idx.size(0))
        if n_struct > 0:
            bank_idx = torch.randint(0, int(mutation_bank.size(0)), (n_struct,), **i64)
            len_p, len_b = torch.empty(n_struct, **i64), torch.empty(n_struct, **i64)
            rand_p = torch.rand(n_struct, **f32)
            rand_b = torch.rand(n_struct, **f32)
            sp_, ep_ = torch.empty(n_struct, **i64), torch.empty(n_struct, **i64)
            sb_, eb_ = torch.empty(n_struct, **i64), torch.empty(n_struct, **i64)
            N.check(lib.ws_subtree_pick(ptr(offspring), ptr(struct_idx), n_struct, L,
                                        ptr(token_arities), vocab, ptr(rand_p), ptr(len_p),
                                        ptr(sp_), ptr(ep_), int(PAD_ID), st))
            N.check(lib.ws_subtree_pick(ptr(mutation_bank), ptr(bank_idx), n_struct, L,
                                        ptr(token_arities), vocab, ptr(rand_b), ptr(len_b),
                                        ptr(sb_), ptr(eb_), int(PAD_ID), st))
            child = torch.empty(n_struct, L, dtype=torch.uint8, device=dev)
            dummy = torch.empty(n_struct, L, dtype=torch.uint8, device=dev)
            N.check(lib.ws_splice_rows(ptr(offspring), ptr(mutation_bank), ptr(struct_idx),
                                       ptr(bank_idx), None, None, ptr(sp_), ptr(ep_), ptr(sb_),
                                       ptr(eb_), None, ptr(child), ptr(dummy), n_struct, L,
                                       int(PAD_ID), None, 0.0, None, st))
            offspring.index_copy_(0, struct_idx, child)
    hoist_idx = torch.nonzero(hoist_mask).squeeze(1)
    n_hoist = int(hoist_idx.size(0))
    if n_hoist > 0:
        r_ints = torch.randint(0, 1000000, (n_hoist,), **i64)
        N.check(lib.ws_hoist_rows(ptr(offspring), ptr(hoist_idx), n_hoist, L, ptr(token_arities),
                                  vocab, ptr(r_ints), int(PAD_ID), st))

    # 4. PSO over the offspring's constants (per-row evaluator, torch RMSE, bests, update)
    final_consts, final_fit = offspring_consts, torch.empty(0, **f32)
    if pso_steps > 0:
        P = int(pso_particles)
        gbest_pos = offspring_consts.clone()
        gbest_err = torch.full((B,), float("inf"), **f32)
        pop_expanded = offspring.repeat_interleave(P, 0)
        pos = offspring_consts.unsqueeze(1).repeat(1, P, 1)
        jitter = torch.randn(B, P - 1, K, **f32) * 1.0
        pos[:, 1:, :] = pos[:, 1:, :] + jitter
        vel = torch.randn_like(pos) * 0.1
        pbest_pos = pos.clone()
        pbest_err = torch.full((B, P), float("inf"), **f32)
        preds = torch.empty(B * P, n_data, **f32)
        sp = torch.empty(B * P * n_data, **i32)
        err_flags = torch.empty(B * P * n_data, dtype=torch.uint8, device=dev)
        ids = (PAD_ID, id_x_start, id_C, id_pi, id_e, id_0, id_1, id_2, id_3, id_4, id_5, id_6,
               id_10, op_add, op_sub, op_mul, op_div, op_pow, op_mod, op_sin, op_cos, op_tan,
               op_log, op_exp, op_sqrt, op_abs, op_neg, op_fact, op_floor, op_ceil, op_sign,
               op_gamma, op_lgamma, op_asin, op_acos, op_atan)
        for _ in range(int(pso_steps)):
            flat_pos = pos.view(-1, K)
            eval_rpn(pop_expanded, X, flat_pos, preds, sp, err_flags, *ids, pi_val, e_val, 0)
            diff = preds - Y_target.unsqueeze(0)
            mse = torch.mean(diff * diff, 1)
            rmse = torch.sqrt(mse)
            rmse = torch.where(torch.isnan(rmse), torch.full_like(rmse, float("inf")), rmse)
            curr = rmse.view(B, P)
            pso_update_bests(curr, pbest_err, pbest_pos, pos, gbest_err, gbest_pos)
            r1 = torch.rand(B, P, K, **f32)
            r2 = torch.rand(B, P, K, **f32)
            pso_update(pos, vel, pbest_pos, gbest_pos, r1, r2, _f32(pso_w), _f32(pso_c1),
                       _f32(pso_c2))
        final_consts, final_fit = gbest_pos, gbest_err
    return [offspring, final_consts, final_fit]
