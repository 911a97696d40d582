"""ctypes binding of libwarpsym.so (the C ABI declared in include/warpsym.h).

The library is loaded from this package directory, or from the path in the environment
variable WARPSYM_LIB (for example the bounds-checked build libwarpsym_bc.so).  There is no
fallback: if the shared library is missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("WARPSYM_LIB") or os.path.join(_PKG_DIR, "libwarpsym.so")
BC_LIB_PATH = os.path.join(_PKG_DIR, "libwarpsym_bc.so")  # the bounds-checked build

WS_OK = 0
WS_F32, WS_F64 = 0, 1
WS_POLICY_FUSED, WS_POLICY_CLASSIC = 0, 1
WS_LOSS_RMSE, WS_LOSS_MSE, WS_LOSS_R2, WS_LOSS_SSE = 0, 1, 2, 3
WS_VALIDATE_KERNEL, WS_VALIDATE_CLAMPED, WS_VALIDATE_STACK = 0, 1, 2


class TokenMap(C.Structure):
    """Mirror of ws_token_map: the reference's scalar token-ID arguments (bindings.cpp:7-27)."""

    _fields_ = [(n, C.c_int32) for n in (
        "pad_id", "id_x_start", "id_C", "id_pi", "id_e",
        "id_0", "id_1", "id_2", "id_3", "id_4", "id_5", "id_6", "id_10",
        "op_add", "op_sub", "op_mul", "op_div", "op_pow", "op_mod",
        "op_sin", "op_cos", "op_tan", "op_log", "op_exp",
        "op_sqrt", "op_abs", "op_neg",
        "op_fact", "op_floor", "op_ceil", "op_sign",
        "op_gamma", "op_lgamma",
        "op_asin", "op_acos", "op_atan")] + [("pi_val", C.c_double), ("e_val", C.c_double)]

    INT_FIELDS = tuple(n for n, _ in _fields_[:-2])

    @classmethod
    def from_args(cls, *ids, pi_val: float, e_val: float) -> "TokenMap":
        """Builds the map from the reference's positional ID arguments (same order)."""
        if len(ids) != len(cls.INT_FIELDS):
            raise TypeError("expected %d token ids, got %d" % (len(cls.INT_FIELDS), len(ids)))
        m = cls()
        for name, v in zip(cls.INT_FIELDS, ids):
            setattr(m, name, int(v))
        m.pi_val = float(pi_val)
        m.e_val = float(e_val)
        return m

    def key(self) -> tuple:
        return tuple(getattr(self, n) for n in self.INT_FIELDS) + (self.pi_val, self.e_val)


WS_PHASE_ALL, WS_PHASE_COMPILE, WS_PHASE_EVALUATE = 0, 1, 2


class SimplifyIds(C.Structure):
    """Mirror of ws_simplify_ids: the simplifier's operator / literal IDs (argument order of
    simplify_kernels.cu:665-678)."""

    _fields_ = [(n, C.c_int32) for n in (
        "op_plus", "op_minus", "op_mult", "op_div", "op_neg", "op_mod", "op_pow",
        "op_sin", "op_cos", "op_tan", "op_asin", "op_acos", "op_atan",
        "op_log", "op_exp", "op_sqrt", "op_abs", "op_gamma", "op_lgamma", "op_floor", "op_ceil",
        "op_sign", "id_0", "id_1", "id_2", "id_3", "id_4", "id_5", "id_6")]


class FitnessOpts(C.Structure):
    _fields_ = [("strict_mode", C.c_int32), ("policy", C.c_int32), ("loss", C.c_int32),
                ("schedule", C.c_int32), ("invalid_value", C.c_double), ("phase", C.c_int32),
                ("reserved", C.c_int32)]


class Problem(C.Structure):
    """ws_problem: one problem of a batched fitness call (device pointers)."""
    _fields_ = [("population", C.c_void_p), ("B", C.c_int64), ("x", C.c_void_p),
                ("num_vars", C.c_int64), ("D", C.c_int64), ("constants", C.c_void_p),
                ("K", C.c_int64), ("y", C.c_void_p), ("out_loss", C.c_void_p),
                ("out_ninvalid", C.c_void_p), ("ids", C.POINTER(TokenMap))]


class GpProblem(C.Structure):
    """ws_gp_problem: one problem of a batched GP generation (device pointers)."""
    _fields_ = [("population", C.c_void_p), ("B", C.c_int64), ("constants", C.c_void_p),
                ("K", C.c_int64), ("fitness", C.c_void_p), ("num_vars", C.c_int64),
                ("ids", C.POINTER(TokenMap)), ("seed", C.c_uint64), ("generation", C.c_uint64)]


class GpOpts(C.Structure):
    _fields_ = [("tournament_size", C.c_int32), ("elitism", C.c_int32),
                ("crossover_rate", C.c_float), ("mutation_rate", C.c_float),
                ("const_mutation_rate", C.c_float), ("const_sigma", C.c_float),
                ("parsimony_eps", C.c_float), ("reserved", C.c_int32)]


class LbfgsOpts(C.Structure):
    """ws_lbfgs_opts: options of the per-program L-BFGS (torch.optim.LBFGS names)."""
    _fields_ = [("max_iter", C.c_int32), ("max_eval", C.c_int32), ("history", C.c_int32),
                ("max_ls", C.c_int32), ("lr", C.c_double), ("tolerance_grad", C.c_double),
                ("tolerance_change", C.c_double), ("grad_clip", C.c_double),
                ("sync_every", C.c_int32), ("reserved", C.c_int32)]


class PointMutation(C.Structure):
    """ws_point_mutation: the Philox point mutation of evolve_generation (device pointers)."""
    _fields_ = [("arities", C.c_void_p), ("vocab", C.c_int32), ("n0", C.c_int32),
                ("n1", C.c_int32), ("n2", C.c_int32), ("ids0", C.c_void_p), ("ids1", C.c_void_p),
                ("ids2", C.c_void_p), ("rate", C.c_float), ("reserved", C.c_int32),
                ("seed", C.c_uint64), ("generation", C.c_uint64)]


_P = C.c_void_p
_I64 = C.c_int64
_I32 = C.c_int32
_SIGS = {
    "ws_version": (C.c_char_p, []),
    "ws_last_error": (C.c_char_p, []),
    "ws_bounds_status": (_I32, [C.POINTER(C.c_int32), C.POINTER(C.c_uint64), _I32]),
    "ws_debug_bounds_selftest": (_I32, [C.POINTER(C.c_uint64)]),
    "ws_fitness_workspace_bytes": (C.c_size_t, [_I64, _I64, _I32]),
    "ws_schedule_count": (_I32, []),
    "ws_eval_rpn": (_I32, [_I32, _P, _I64, _I64, _P, _I64, _I64, _P, _I64, _P, _P, _P,
                           C.POINTER(TokenMap), _I32, _P]),
    "ws_eval_rpn_fused": (_I32, [_I32, _P, _I64, _I64, _P, _I64, _I64, _P, _I64, _P, _P,
                                 C.POINTER(TokenMap), _I32, _I32, _P, C.c_size_t, _P]),
    "ws_eval_fitness": (_I32, [_I32, _P, _I64, _I64, _P, _I64, _I64, _P, _I64, _P, _P, _P,
                               C.POINTER(TokenMap), C.POINTER(FitnessOpts), _P, C.c_size_t, _P]),
    "ws_eval_fitness_static": (_I32, [_I32, _P, _I64, _I64, _P, _I64, _I64, _P, _I64, _P, _P,
                                      _P, C.POINTER(TokenMap), C.POINTER(FitnessOpts), _P]),
    "ws_static_scratch_bytes": (C.c_size_t, []),
    "ws_batch_workspace_bytes": (_I32, [_I32, _P, _I32, _I64, C.POINTER(FitnessOpts),
                                        C.POINTER(C.c_size_t)]),
    "ws_batch_create": (_I32, [_I32, _P, _I32, _I64, C.POINTER(FitnessOpts), _P, C.c_size_t,
                               _P, C.POINTER(_P)]),
    "ws_batch_eval": (_I32, [_P, _I32, _P]),
    "ws_batch_info": (_I64, [_P, _I32]),
    "ws_batch_set_cancel": (_I32, [_P, _P]),
    "ws_batch_destroy": (None, [_P]),
    "ws_gp_workspace_bytes": (_I32, [_I32, _P, _I32, _I64, C.POINTER(C.c_size_t)]),
    "ws_gp_create": (_I32, [_I32, _P, _I32, _I64, C.POINTER(GpOpts), _P, C.c_size_t, _P,
                            C.POINTER(_P)]),
    "ws_gp_step": (_I32, [_P, _P]),
    "ws_gp_set_generation": (_I32, [_P, C.c_uint64, _P]),
    "ws_gp_destroy": (None, [_P]),
    "ws_mutate_population": (_I32, [_P, _I64, _I64, _P, _P, _P, _I64, _P, _I64, _P, _I64, _P,
                                    _I64, C.c_float, _I32, _P]),
    "ws_crossover_splicing": (_I32, [_P, _P, _I64, _I64, _P, _P, _P, _P, _P, _P, _I32, _P, _P]),
    "ws_constant_perturbation": (_I32, [_I32, _P, _I64, _I64, C.c_float, C.c_float, C.c_float,
                                        C.c_float, C.c_uint32, _P]),
    "ws_generate_random_rpn": (_I32, [_P, _I64, _I64, _P, _I64, _P, _I64, _P, _I64, C.c_uint64,
                                      C.c_float, C.c_float, C.c_float, _P]),
    "ws_update_best": (_I32, [_P, _I64, _I64, _P, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _I32,
                              C.c_float, _P]),
    "ws_check_improvement": (_I32, [_P, _I64, _P, _P, C.c_float, _P]),
    "ws_batch_update_best": (_I32, [_P, _I64, _I64, _P, _I64, _P, _P, _P, _P, _P, C.c_float, _P]),
    "ws_population_hashes": (_I32, [_P, _I64, _I64, _P, _P, _I32, _I32, _I32, _P]),
    "ws_structural_dedup": (_I32, [_P, _I64, _P, _P, _P, _P]),
    "ws_count_unique": (_I32, [_P, _I64, _P, _P]),
    "ws_replacement_positions": (_I32, [_P, _I64, _P, _P, _P]),
    "ws_fitness_sharing_penalty": (_I32, [_P, _I64, _I64, _I32, _I32, _I32, _I32, _P, _P, _P, _P]),
    "ws_dedup_table_slots": (_I64, []),
    "ws_sharing_table_slots": (_I64, []),
    "ws_eval_rpn_backward": (_I32, [_I32, _P, _I64, _I64, _P, _I64, _I64, _P, _I64, _P, _P,
                                    C.POINTER(TokenMap), _P]),
    "ws_eval_rpn_backward_workspace_bytes": (_I32, [_I64, C.POINTER(C.c_size_t)]),
    "ws_eval_rpn_backward_ws": (_I32, [_I32, _P, _I64, _I64, _P, _I64, _I64, _P, _I64, _P, _P,
                                       C.POINTER(TokenMap), _P, C.c_size_t, _P]),
    "ws_subtree_pick": (_I32, [_P, _P, _I64, _I64, _P, _I32, _P, _P, _P, _P, _I32, _P]),
    "ws_splice_valid": (_I32, [_P, _P, _P, _P, _P, _P, _P, _P, _I64, _I64, _P]),
    "ws_splice_rows": (_I32, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I64, _I64,
                              _I32, _P, C.c_float, C.POINTER(PointMutation), _P]),
    "ws_mutate_rows": (_I32, [_P, _P, _I64, _I64, _P, C.c_float, C.POINTER(PointMutation), _I32,
                              _P]),
    "ws_sbx_constants": (_I32, [_P, _P, _P, _P, _P, _P, _P, _I64, _I64, C.c_float, _P]),
    "ws_splice_constants": (_I32, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I64,
                                   _I64, _I64, _I32, _P]),
    "ws_hoist_rows": (_I32, [_P, _P, _I64, _I64, _P, _I32, _P, _I32, _P]),
    "ws_loss_grad_workspace_bytes": (_I32, [_I32, _I64, _I64, _I64, _I64, _I64,
                                            C.POINTER(C.c_size_t)]),
    "ws_loss_grad": (_I32, [_I32, _P, _I64, _I64, _P, _I64, _I64, _P, _I64, _P, _P, _P, _P,
                            C.POINTER(TokenMap), _P, C.c_size_t, _P]),
    "ws_lbfgs_adjoint_workspace_bytes": (_I32, [_I32, _I64, _I64, _I64, _I64, _I64, _I32,
                                                C.POINTER(C.c_size_t)]),
    "ws_lbfgs_adjoint": (_I32, [_I32, _P, _I64, _I64, _P, _I64, _I64, _P, _I64, _P,
                                C.POINTER(LbfgsOpts), _P, _P, C.POINTER(TokenMap), _P,
                                C.c_size_t, _P]),
    "ws_decode_rpn": (_I32, [_P, _I64, _I64, _P, _I32, _I64, C.POINTER(C.c_char_p), _I64, _P,
                             _I64, _I32, _I32, _P, C.c_size_t, _P, C.POINTER(C.c_size_t)]),
    "ws_pso_update": (_I32, [_I32, _P, _P, _P, _P, _P, _P, C.c_float, C.c_float, C.c_float,
                             _I64, _I64, _I64, _P]),
    "ws_pso_update_bests": (_I32, [_I32, _P, _P, _P, _P, _P, _P, _I64, _I64, _I64, _P]),
    "ws_fused_pso": (_I32, [_I32, _P, _I64, _I64, _P, _I64, _P, _I64, _I64, _P, _P, _P, _I32,
                            _I32, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float,
                            C.POINTER(TokenMap), C.c_uint64, _P]),
    "ws_lbfgs_optimize": (_I32, [_I32, _P, _I64, _I64, _P, _I64, _P, _I64, _I64, _P, _P, _I32,
                                 _I32, C.c_float, C.c_float, C.c_float, C.POINTER(TokenMap), _P]),
    "ws_simplify_batch": (_I32, [_P, _I64, _I64, _P, _I64, _P, _P, _P, _I64, _I32,
                                 C.POINTER(SimplifyIds), _P]),
    "ws_validate_rpn_batch": (_I32, [_P, _I32, _I64, _I64, _P, _I64, _I32, _I32, _P, _P]),
    "ws_find_subtree_ranges": (_I32, [_P, _I64, _I64, _P, _I64, _I32, _P, _P, _P]),
    "ws_precompute_subtree_starts": (_I32, [_P, _I64, _I64, _P, _I64, _P, _P]),
    "ws_tournament_select": (_I32, [_P, _I64, _P, _I64, _P, _I64, _P, _P, _P, _P, _P]),
    "ws_tournament_select_offsets": (_I32, [_P, _I64, _P, _I64, _P, _I64, _P, _P, _P, _I32, _I32,
                                            _P, _P]),
    "ws_debug_token_lut": (_I32, [C.POINTER(TokenMap), _I64, _I32, _P, _P]),
    "ws_debug_compile": (_I32, [_I32, _P, _I64, _P, _I64, C.POINTER(TokenMap), _I64, _I32, _I32,
                                _P, _P, _P]),
    "ws_debug_run_tape": (_I32, [_I32, _P, _P, _I32, _P, _I64, _I32, _P, _P]),
    "ws_debug_compile_agree": (_I32, [_I32, _P, _I64, _I64, _P, _I64, C.POINTER(TokenMap),
                                      _I64, _I32, _I32, _I32, _P]),
}

_lib = None
_lock = threading.Lock()


def lib():
    """Loads libwarpsym.so once (raises OSError/RuntimeError when it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    "libwarpsym.so not found at %s: build it with __graft_entry__.build() "
                    "(there is no CPU fallback)" % LIB_PATH)
            handle = C.CDLL(LIB_PATH)
            for name, (res, args) in _SIGS.items():
                fn = getattr(handle, name)
                fn.restype = res
                fn.argtypes = args
            _lib = handle
    return _lib


def bounds_status(reset: bool = False):
    """(enabled, word): whether the loaded library is the bounds-checked build, and its first
    recorded out-of-range index ((site << 32) | index; 0 when none)."""
    en, w = C.c_int32(0), C.c_uint64(0)
    check(lib().ws_bounds_status(C.byref(en), C.byref(w), 1 if reset else 0))
    return bool(en.value), int(w.value)


def check(status: int) -> None:
    """Raises RuntimeError carrying the library's message when status != WS_OK."""
    if status != WS_OK:
        msg = lib().ws_last_error().decode("utf-8", "replace")
        raise RuntimeError(msg or "warpsym error %d" % status)


def exported_symbols() -> list:
    return sorted(_SIGS)
