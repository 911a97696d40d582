"""Multi-process (N > 1) host logic on CPU: world_size-2 gloo process groups.

Each rank scores its own contiguous shard with the CPU oracle standing in for the GPU evaluator
(no GPU here); the gathered fitness must equal a single-process evaluation of the whole
population, for populations that do not divide evenly and for fewer programs than ranks; the
timing reduction takes the maximum over ranks."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import ws_testlib as tl


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _case():
    rng = np.random.default_rng(11)
    g = tl.GPUGrammar(num_variables=2, operators=tl.C1_OPERATORS)
    pop, consts = tl.random_population(g, 257, 24, 4, rng, valid_only=False)
    X = rng.uniform(-3, 3, size=(2, 64)).astype(np.float32)
    y = (X[0] * X[1]).astype(np.float32)
    return g, pop, consts, X, y


def _worker(rank, world, port, n_programs, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from warpsymbolic_b200.sharding import ShardedEvaluator, max_over_ranks, shard_bounds
        g, pop, consts, X, y = _case()
        pop, consts = pop[:n_programs], consts[:n_programs]
        tm = tl.token_map(g)

        def score(p, c):
            if len(p) == 0:
                return torch.empty(0, dtype=torch.float32)
            return torch.from_numpy(tl.oracle.fitness(tm, p.numpy(), X, c.numpy(), y,
                                                      policy="classic", loss="rmse"))

        ev = ShardedEvaluator(score)
        full = ev.evaluate(torch.from_numpy(pop), torch.from_numpy(consts))
        local, (s, e) = ev.evaluate_local(torch.from_numpy(pop), torch.from_numpy(consts))
        t = max_over_ranks(0.5 + rank)
        q.put((rank, full.numpy(), (s, e), shard_bounds(n_programs, world, rank), t))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n_programs", [257, 1])
def test_two_rank_sharded_evaluation_matches_single_process(n_programs):
    g, pop, consts, X, y = _case()
    want = tl.oracle.fitness(tl.token_map(g), pop[:n_programs], X, consts[:n_programs], y,
                             policy="classic", loss="rmse")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, n_programs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    bounds = {}
    for rank, full, se, sb, t in res:
        np.testing.assert_array_equal(full, want)
        assert se == sb
        bounds[rank] = se
        assert t == 1.5
    assert bounds[0][0] == 0 and bounds[0][1] == bounds[1][0] and bounds[1][1] == n_programs


def test_shard_bounds_partition():
    from warpsymbolic_b200.sharding import shard_bounds
    for n in (0, 1, 7, 1 << 20):
        for world in (1, 2, 3, 8):
            b = [shard_bounds(n, world, r) for r in range(world)]
            assert b[0][0] == 0 and b[-1][1] == n
            assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
            sizes = [e - s for s, e in b]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_bounds(10, 2, 2)


# ---- row sharding -----------------------------------------------------------------------
def _row_case(dtype):
    rng = np.random.default_rng(12)
    g = tl.GPUGrammar(num_variables=3, operators=tl.C1_OPERATORS)
    pop, consts = tl.random_population(g, 300, 24, 4, rng, valid_only=False)
    X = rng.uniform(-3, 3, size=(3, 1001)).astype(dtype)
    y = (np.sin(X[0]) + X[1] * X[2]).astype(dtype)
    return g, pop, consts.astype(dtype), X, y


def _row_worker(rank, world, port, dtype_name, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from warpsymbolic_b200.sharding import RowShardedEvaluator, shard_bounds
        dtype = np.dtype(dtype_name)
        g, pop, consts, X, y = _row_case(dtype)
        tm = tl.token_map(g)
        s, e = shard_bounds(X.shape[1], world, rank)

        def partial(p, xs, ys, c):  # the oracle stands in for the GPU evaluator
            sse, ninv = tl.oracle.fitness(tm, p.numpy(), xs.numpy(), c.numpy(), ys.numpy(),
                                          policy="classic", loss="sse", with_ninv=True)
            return torch.from_numpy(sse), torch.from_numpy(ninv)

        ev = RowShardedEvaluator(partial_fn=partial)
        out = {}
        for loss in ("mse", "rmse", "r2"):
            out[loss] = ev.evaluate(torch.from_numpy(pop), torch.from_numpy(X[:, s:e].copy()),
                                    torch.from_numpy(y[s:e].copy()), torch.from_numpy(consts),
                                    loss=loss).numpy()
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("dtype_name", ["float32", "float64"])
def test_two_rank_row_sharding_matches_single_process(dtype_name):
    dtype = np.dtype(dtype_name)
    g, pop, consts, X, y = _row_case(dtype)
    tm = tl.token_map(g)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_row_worker, args=(r, 2, port, dtype_name, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for loss in ("mse", "rmse", "r2"):
        want = tl.oracle.fitness(tm, pop, X, consts, y, policy="classic", loss=loss)
        a, b = res[0][loss], res[1][loss]
        np.testing.assert_array_equal(a, b)  # every rank forms the same losses
        inv = 1e15 if dtype == np.float32 else 1e100
        bad = np.abs(want) >= inv * 0.5
        assert (np.abs(a) >= inv * 0.5).tolist() == bad.tolist(), loss
        rtol = 1e-6 if dtype == np.float32 else 1e-12
        # R^2 = 1 - MSE / Var(y) cancels near 0: an absolute floor of a few ulps of 1
        atol = 0.0 if loss != "r2" else (1e-6 if dtype == np.float32 else 1e-14)
        np.testing.assert_allclose(a[~bad], want[~bad], rtol=rtol, atol=atol)
        assert (~bad).sum() > 100


# ---- failure detection: a rank whose evaluator fails ----------------------------------------
def _failing_worker(rank, world, port, q):
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    # a short process-group timeout bounds how long the healthy rank can wait for the failed one
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=10))
    try:
        from warpsymbolic_b200.sharding import ShardedEvaluator
        g, pop, consts, X, y = _case()
        tm = tl.token_map(g)

        def score(p, c):
            if rank == 1:
                raise RuntimeError("injected evaluator failure")
            return torch.from_numpy(tl.oracle.fitness(tm, p.numpy(), X, c.numpy(), y,
                                                      policy="classic", loss="rmse"))

        try:
            ShardedEvaluator(score).evaluate(torch.from_numpy(pop), torch.from_numpy(consts))
            q.put((rank, "completed"))
        except Exception as e:  # the failure, as each rank sees it
            q.put((rank, "%s: %s" % (type(e).__name__, str(e)[:200])))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def test_a_failing_rank_ends_the_sharded_evaluation_with_an_error():
    """Rank 1's evaluator raises before the gather (a host-made failure); rank 1 reports it and
    leaves; rank 0's gather then ends with an error (peer closed, or the process group's 10 s
    timeout) instead of waiting: both ranks report an error and exit."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_failing_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
        assert not p.is_alive()
    assert "injected evaluator failure" in res[1], res
    assert res[0] != "completed", res
