"""Token vocabulary of the RPN bytecode (mirror of src/warpsymbolic/gpu/grammar.py).

IDs are assigned exactly as the reference assigns them (grammar.py:18-174): PAD = 0, then the
active variables x0..x{V-1}, then the terminals C, 0, 1, 2, 3, 4, 5, 6, 10, pi, e, then the
enabled operators in a fixed order with `sqrt`, `abs` and the always-present `neg` last.  The
reference reads the operator toggles from its global config (config.py:119-142); here they are
an explicit argument whose default equals that config's defaults.
"""
from __future__ import annotations

from typing import Dict, Iterable, List, Optional

PAD_ID = 0

# Arity of every operator the bytecode knows (reference symbolic/grammar.py OPERATORS).
OPERATORS: Dict[str, int] = {
    '+': 2, '-': 2, '*': 2, '/': 2, 'pow': 2, '%': 2,
    'sin': 1, 'cos': 1, 'tan': 1, 'asin': 1, 'acos': 1, 'atan': 1,
    'log': 1, 'exp': 1, 'sqrt': 1, 'abs': 1, 'neg': 1,
    'floor': 1, 'ceil': 1, 'sign': 1, 'fact': 1, 'gamma': 1, 'lgamma': 1,
}

# Order in which enabled operators receive IDs (grammar.py:53-87).
_OPERATOR_ORDER = ['+', '-', '*', '/', 'pow', '%', 'sin', 'cos', 'tan', 'log', 'exp', 'fact',
                   'gamma', 'lgamma', 'asin', 'acos', 'atan', 'floor', 'ceil', 'sign']

# GpuGlobals defaults (config.py:119-142): pow, sqrt, abs on; %, tan, fact, gamma, lgamma,
# asin, acos, atan, floor, ceil, sign off; neg always on.
DEFAULT_OPERATORS = ('+', '-', '*', '/', 'pow', 'sin', 'cos', 'log', 'exp', 'sqrt', 'abs')

TERMINALS_AFTER_VARS = ['C', '0', '1', '2', '3', '4', '5', '6', '10', 'pi', 'e']

# Literal values passed by the reference VM (cuda_vm.py:148, 171).
PI_VAL = 3.14159265359
E_VAL = 2.718281828


class GPUGrammar:
    def __init__(self, num_variables: int = 1, operators: Optional[Iterable[str]] = None):
        ops = set(DEFAULT_OPERATORS if operators is None else operators)
        unknown = ops - set(OPERATORS)
        if unknown:
            raise ValueError("unknown operators: %s" % sorted(unknown))
        self.token_to_id: Dict[str, int] = {'<PAD>': PAD_ID}
        self.id_to_token: Dict[int, str] = {PAD_ID: '<PAD>'}
        self.next_id = 1
        if num_variables > 1:
            self.active_variables = ['x%d' % i for i in range(num_variables)]
        else:
            self.active_variables = ['x0']
        self.terminals = self.active_variables + TERMINALS_AFTER_VARS
        for t in self.terminals:
            self._add(t)
        self.operators: List[str] = [op for op in _OPERATOR_ORDER if op in ops]
        if 'sqrt' in ops:
            self.operators.append('sqrt')
        if 'abs' in ops:
            self.operators.append('abs')
        self.operators.append('neg')
        for op in self.operators:
            self._add(op)
        self.vocab_size = self.next_id
        if self.vocab_size > 255:
            raise ValueError("Vocabulary size %d exceeds uint8 limit (255)." % self.vocab_size)
        self.op_ids = {op: self.token_to_id[op] for op in self.operators}
        self.token_arity = {op: OPERATORS.get(op, 1) for op in self.operators}

    def _add(self, name: str) -> None:
        self.token_to_id[name] = self.next_id
        self.id_to_token[self.next_id] = name
        self.next_id += 1

    # ---- helpers used by the evaluator -----------------------------------------------------
    def scalar_ids(self) -> tuple:
        """The reference's positional ID arguments (cuda_vm.py:34-82, bindings.cpp:7-27):
        PAD_ID, id_x_start, id_C, id_pi, id_e, id_0..id_6, id_10, op_add ... op_atan."""
        g = self.token_to_id
        get = lambda k, d: g.get(k, d)
        return (
            get('<PAD>', -999), get(self.active_variables[0], -999),
            get('C', -1), get('pi', -100), get('e', -100),
            get('0', -1), get('1', -1), get('2', -1), get('3', -1), get('4', -1), get('5', -1),
            get('6', -1), get('10', -1),
            get('+', -100), get('-', -100), get('*', -100), get('/', -100), get('pow', -100),
            get('%', -100),
            get('sin', -100), get('cos', -100), get('tan', -100), get('log', -100),
            get('exp', -100),
            get('sqrt', -100), get('abs', -100), get('neg', -100),
            get('fact', -100), get('floor', -100), get('ceil', -100), get('sign', -100),
            get('gamma', -100), get('lgamma', -100),
            get('asin', -100), get('acos', -100), get('atan', -100),
        )

    def arities(self) -> List[int]:
        """Arity per token ID (terminals 0), like get_arity_tensor (grammar.py:206-219)."""
        a = [0] * self.vocab_size
        for op in self.operators:
            a[self.token_to_id[op]] = self.token_arity[op]
        return a

    def get_arity_tensor(self, device=None):
        import torch
        return torch.tensor(self.arities(), dtype=torch.int32, device=device)

    def encode(self, tokens: Iterable[str], length: int) -> List[int]:
        """RPN token names -> PAD-terminated, left-packed uint8 row of `length`."""
        ids = [self.token_to_id[t] for t in tokens]
        if len(ids) > length:
            raise ValueError("program longer than %d" % length)
        return ids + [PAD_ID] * (length - len(ids))
