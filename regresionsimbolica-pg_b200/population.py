"""Population maintenance of the reference's GPUOperators, on this library's kernels.

`PopulationOperators` restates the methods of `GPUOperators` (src/warpsymbolic/gpu/operators.py)
that create and repair individuals:

  * the token tables (`_init_arity_masks`, operators.py:63-149): arities per token ID, the
    terminal IDs, and the operator IDs repeated round(200 * prior) times so that the native
    generator's uniform draw follows the configured per-operator prior;
  * the native seed sequence (`_next_native_seed`, :46-49): seed_k = (torch.initial_seed() at
    construction + k * 0x9E3779B97F4A7C15 + salt) mod 2^63;
  * the category weights of the generator (`_sampling_category_weights`, :206-236, the "full"
    sampling profile);
  * `generate_random_population` (:360-420): `generate_random_rpn` with the next seed (salt
    0xA341316C), then `_force_multi_variable` (:238-330);
  * `repair_invalid_population` (:1496-1525): stack validation, fresh random individuals in the
    invalid rows, fresh constants U[CONSTANT_MIN_VALUE, CONSTANT_MAX_VALUE] (or integers) drawn
    with the torch generator in the reference's order.

With the same torch seed and the same configuration the results are the reference's, bit for
bit: the kernels reproduce the reference extension's outputs and the torch draws are made in the
same order with the same shapes.  The configuration keys and defaults are those of the
reference's `GpuGlobals` (src/warpsymbolic/gpu/config.py) that these methods read.
"""
from __future__ import annotations

from typing import Dict, Optional, Tuple

import torch

from . import rpn_cuda_native as _rn
from .grammar import GPUGrammar, OPERATORS, PAD_ID

# The reference's defaults for the keys these methods read (config.py:134-140, 220-225, 268).
DEFAULT_CONFIG: Dict[str, object] = {
    "OPERATOR_WEIGHT_BY_NAME": {
        '+': 0.20, '-': 0.20, '*': 0.20, '/': 0.15, 'pow': 0.10, '%': 0.02,
        'sin': 0.10, 'cos': 0.10, 'tan': 0.05, 'log': 0.08, 'exp': 0.08,
        'fact': 0.08, 'floor': 0.01, '__gamma_family__': 0.08,
        'asin': 0.01, 'acos': 0.01, 'atan': 0.01, 'ceil': 0.005,
        'sign': 0.005, 'sqrt': 0.10, 'abs': 0.05, 'neg': 0.02,
    },
    "NEG_OPERATOR_WEIGHT": 0.02,
    "TERMINAL_VS_VARIABLE_PROB": 0.40,
    "CONSTANT_MIN_VALUE": -25.0,
    "CONSTANT_MAX_VALUE": 25.0,
    "CONSTANT_INT_MIN_VALUE": -25,
    "CONSTANT_INT_MAX_VALUE": 25,
    "FORCE_INTEGER_CONSTANTS": False,
    "VAR_FORCE_SEED_PERCENT": 0.0,
}

# Operators in the order of the reference's prior table (operators.py:90-95).
_PRIOR_ORDER = ('+', '-', '*', '/', 'pow', '%', 'sin', 'cos', 'tan', 'log', 'exp', 'fact',
                'floor', '__gamma_family__', 'asin', 'acos', 'atan', 'ceil', 'sign', 'sqrt',
                'abs')
_SEED_STEP = 0x9E3779B97F4A7C15
_MASK63 = 0x7FFFFFFFFFFFFFFF
_GENERATE_SALT = 0xA341316C


class PopulationOperators:
    """Random generation and repair of RPN populations with the reference's semantics.

    `grammar` gives the token IDs (the reference's GPUGrammar numbering); `config` overrides keys
    of DEFAULT_CONFIG.  The seed sequence starts from torch.initial_seed() when the object is
    created, as the reference's GPUOperators does."""

    def __init__(self, grammar: GPUGrammar, device, max_len: int, num_variables: int,
                 dtype: torch.dtype = torch.float32, config: Optional[Dict[str, object]] = None):
        self.grammar = grammar
        self.device = torch.device(device)
        self.max_len = int(max_len)
        self.num_variables = int(num_variables)
        self.dtype = dtype
        self.config = dict(DEFAULT_CONFIG)
        self.config.update(config or {})
        self._rng_seed = int(torch.initial_seed()) & _MASK63
        self._rng_counter = 0
        g = grammar
        self.token_arity = torch.zeros(g.vocab_size + 1, dtype=torch.long, device=self.device)
        arity_0, arity_1, arity_2 = [], [], []
        for t in g.terminals:
            arity_0.append(g.token_to_id[t])
        for op in g.operators:
            tid = g.token_to_id[op]
            a = OPERATORS.get(op, 1)
            self.token_arity[tid] = a
            (arity_1 if a == 1 else arity_2 if a == 2 else []).append(tid)
        prior_map = self.config["OPERATOR_WEIGHT_BY_NAME"]
        prior = {name: max(0.0, float(prior_map.get(name, 0.0))) for name in _PRIOR_ORDER}
        gamma = prior.pop('__gamma_family__', 0.0)
        enabled_gamma = [n for n in ('gamma', 'lgamma') if n in g.operators]
        for n in enabled_gamma:
            prior[n] = gamma / len(enabled_gamma)
        prior.setdefault('neg', float(self.config["NEG_OPERATOR_WEIGHT"]))
        self.prior = prior

        def weighted(ids):
            out = []
            for tid in ids:
                w = prior.get(g.id_to_token[int(tid)], 0.0)
                if w > 0.0:
                    out.extend([tid] * max(1, int(round(w * 200.0))))
            return out if out else list(ids)

        u8 = dict(device=self.device, dtype=torch.uint8)
        self.terminal_ids = torch.tensor([g.token_to_id[t] for t in g.terminals], **u8)
        self.arity_0_ids = torch.tensor(arity_0, **u8)
        self.arity_1_ids = torch.tensor(weighted(arity_1), **u8)
        self.arity_2_ids = torch.tensor(weighted(arity_2), **u8)
        self._uniform_arity_1 = list(arity_1)
        self._uniform_arity_2 = list(arity_2)
        self._empty_ids = torch.empty(0, **u8)
        self.token_arity_int = self.token_arity.to(torch.int32)

    # -- seeds and weights ---------------------------------------------------------------------
    def next_native_seed(self, salt: int = 0) -> int:
        seed = (self._rng_seed + self._rng_counter * _SEED_STEP + int(salt)) & _MASK63
        self._rng_counter += 1
        return seed

    def category_weights(self) -> Tuple[float, float, float]:
        """(terminal, unary, binary) category probabilities of the generator."""
        g = self.grammar
        bin_sum = sum(self.prior.get(g.id_to_token[t], 0.0) for t in set(self._uniform_arity_2))
        una_sum = sum(self.prior.get(g.id_to_token[t], 0.0) for t in set(self._uniform_arity_1))
        t_frac = float(self.config["TERMINAL_VS_VARIABLE_PROB"])
        op_sum = max(bin_sum + una_sum, 1e-6)
        t_frac = max(0.05, min(0.95, t_frac))
        o_frac = 1.0 - t_frac
        return t_frac, float(o_frac * una_sum / op_sum), float(o_frac * bin_sum / op_sum)

    # -- generation ------------------------------------------------------------------------------
    def validate(self, population: torch.Tensor) -> torch.Tensor:
        """Stack validity of every row (the generation's validation kernel)."""
        valid = torch.empty(population.shape[0], dtype=torch.bool, device=self.device)
        _rn.validate_rpn_batch(population, self.token_arity_int, valid, PAD_ID)
        return valid

    def generate_random_population(self, size: int) -> torch.Tensor:
        population = torch.empty(size, self.max_len, dtype=torch.uint8, device=self.device)
        seed = self.next_native_seed(_GENERATE_SALT)
        u_ids = self.arity_1_ids if self.arity_1_ids.numel() > 0 else self._empty_ids
        b_ids = self.arity_2_ids if self.arity_2_ids.numel() > 0 else self._empty_ids
        tw, uw, bw = self.category_weights()
        _rn.generate_random_rpn(population, self.terminal_ids.contiguous(), u_ids.contiguous(),
                                b_ids.contiguous(), seed, tw, uw, bw)
        return self.force_multi_variable(population)

    def force_multi_variable(self, population: torch.Tensor) -> torch.Tensor:
        """The reference's variable-forcing pass on its native path.  It picks, for the first
        VAR_FORCE_SEED_PERCENT of the rows and each variable they lack, a random terminal position
        to overwrite; the writes land in tensors that advanced indexing copied, so the
        population comes back unchanged while the torch generator advances by the draws.  Both
        effects are reproduced: rows are left as they are, the same random draws are made."""
        pct = float(self.config["VAR_FORCE_SEED_PERCENT"])
        if self.num_variables <= 1 or pct <= 0:
            return population
        n_force = int(population.shape[0] * pct)
        if n_force < 1:
            return population
        subset = population[:n_force]
        presence = torch.empty(n_force, dtype=torch.int32, device=self.device)
        id_x0 = self.grammar.token_to_id.get('x0', self.grammar.token_to_id.get('x', 1))
        _rn.compute_var_presence(subset, presence, PAD_ID, id_x0, self.num_variables)
        for vi in range(self.num_variables):
            vid = self.grammar.token_to_id.get('x%d' % vi, -1)
            if vid <= 0:
                continue
            bit = 1 << vi
            missing = (presence & bit) == 0
            if int(missing.sum().item()) == 0:
                continue
            missing_idx = missing.nonzero(as_tuple=True)[0]
            rows = subset[missing_idx]  # a copy, as in the reference
            is_term = torch.zeros_like(rows, dtype=torch.bool)
            for tid in self.arity_0_ids:
                is_term |= rows == tid.item()
            has_any = is_term.any(dim=1)
            if not has_any.any():
                continue
            valid_idx = has_any.nonzero(as_tuple=True)[0]
            sel = rows[valid_idx]
            term = is_term[valid_idx]
            pos = (torch.rand_like(term.float()) * term.float()).argmax(dim=1)
            sel[torch.arange(valid_idx.shape[0], device=self.device), pos] = vid
            rows[valid_idx] = sel
            presence[missing_idx[valid_idx]] |= bit
        return population

    def repair_invalid_population(self, population: torch.Tensor,
                                  constants: Optional[torch.Tensor] = None):
        """Replaces every row that fails stack validation by a fresh random individual and
        draws fresh constants for those rows.  Returns (population, constants, n_invalid);
        valid rows are untouched, both tensors are updated in place."""
        invalid_idx = (~self.validate(population)).nonzero(as_tuple=True)[0]
        n_invalid = invalid_idx.numel()
        if n_invalid == 0:
            return population, constants, 0
        population[invalid_idx] = self.generate_random_population(n_invalid)
        if constants is not None and constants.numel() > 0:
            k = constants.shape[1]
            if self.config["FORCE_INTEGER_CONSTANTS"]:
                fresh = torch.randint(int(self.config["CONSTANT_INT_MIN_VALUE"]),
                                      int(self.config["CONSTANT_INT_MAX_VALUE"]) + 1, (n_invalid, k),
                                      device=self.device, dtype=torch.long).to(self.dtype)
            else:
                fresh = torch.empty(n_invalid, k, device=self.device, dtype=self.dtype).uniform_(
                    float(self.config["CONSTANT_MIN_VALUE"]),
                    float(self.config["CONSTANT_MAX_VALUE"]))
            constants[invalid_idx] = fresh
        return population, constants, n_invalid
