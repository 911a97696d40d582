"""Serving loop: every request's result is the same served alone, in the mix, under a memory
budget that admits one request at a time, and on the one-request-at-a-time plain path; requests
that arrive while others run are admitted as slots free up."""
import numpy as np
import pytest
import torch

import ws_testlib  # noqa: F401  (registers the package as warpsymbolic_b200)

pytestmark = pytest.mark.gpu


def _stream():
    from warpsymbolic_b200 import synthetic
    return synthetic.serving_stream(seed=3, n_requests=6, rate=1e6, rows=(300, 4000),
                                    population=256, generations=4, L=32, K=4)


def _same(a, b):
    assert a.kind == b.kind and a.rid == b.rid
    if a.kind == "evaluate":
        assert np.array_equal(a.losses, b.losses, equal_nan=True)
    else:
        assert a.generations == b.generations
        assert a.best_loss == b.best_loss
        assert np.array_equal(a.best_program, b.best_program)
        assert np.array_equal(a.best_constants, b.best_constants)


def test_results_same_alone_in_the_mix_and_plain():
    from warpsymbolic_b200.serving import ContinuousBatchingServer, serve_plain
    reqs = _stream()
    assert {r.kind for r in reqs} == {"fit", "evaluate"}
    srv = ContinuousBatchingServer()
    mixed = srv.serve(reqs, realtime=False)
    assert srv.stats["max_active"] == len(reqs)  # all admitted together
    for r, m in zip(reqs, mixed):
        alone = ContinuousBatchingServer().serve([r], realtime=False)[0]
        _same(m, alone)
    plain = serve_plain(reqs, realtime=False)
    for m, p in zip(mixed, plain):
        _same(m, p)
    fits = [m for m in mixed if m.kind == "fit"]
    assert all(np.isfinite(f.best_loss) and f.best_loss < 1e15 for f in fits)


def test_memory_budget_admits_in_order():
    from warpsymbolic_b200.serving import ContinuousBatchingServer, footprint
    reqs = _stream()
    free = ContinuousBatchingServer().serve(reqs, realtime=False)
    srv = ContinuousBatchingServer(hbm_budget=max(footprint(r) for r in reqs))
    tight = srv.serve(reqs, realtime=False)
    assert srv.stats["max_active"] == 1
    for a, b in zip(free, tight):
        _same(a, b)
    # FIFO: each request is admitted no earlier than the one before it
    adm = [r.admitted for r in sorted(tight, key=lambda q: q.rid)]
    assert all(x <= y for x, y in zip(adm, adm[1:]))
