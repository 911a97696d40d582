"""Host side of the batched path (no GPU): the ctypes ws_problem layout matches the header and
the batched-instances workload has the configured shapes and distributions."""
import ctypes as C

import numpy as np

import ws_testlib as tl


def test_problem_struct_layout():
    P = tl.N.Problem
    assert C.sizeof(P) == 88
    offs = {n: getattr(P, n).offset for n, _ in P._fields_}
    assert offs["population"] == 0 and offs["B"] == 8 and offs["ids"] == 80


def test_batched_workload_shapes():
    from warpsymbolic_b200 import synthetic
    wl = synthetic.batched_workload(seed=1, n_problems=12, programs=64)
    assert len(wl.problems) == 12
    for p in wl.problems:
        V, D = p.X.shape
        assert 1 <= V <= 10 and 100 <= D <= 100_000
        assert p.population.shape == (64, 64) and p.constants.shape == (64, 8)
        assert np.all(np.abs(p.X) <= 4.0) and np.all(np.isfinite(p.y))
        assert len(p.grammar.active_variables) == V
        n = p.n_tokens()
        assert n.min() >= 3 and n.max() <= 64
    assert wl.n_node_evals() > 0
