"""Batched fitness (many problems, one launch sequence): every problem's losses are those of a
single-problem ws_eval_fitness call on it with the same schedule, bit for bit, for uneven
programs, rows, variable counts and vocabularies, and do not depend on the other problems; FP64 exact-operator
batches agree with the CPU oracle; a captured CUDA graph replays the whole pipeline after the
populations are rewritten in place; a cancel flag stops a launch without any wait and leaves the
next launch exact; the autotuner picks a runnable schedule."""
import numpy as np
import pytest
import torch

import ws_testlib as tl

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0") if torch.cuda.is_available() else None
EXACT_OPERATORS = ('+', '-', '*', '/', '%', 'sqrt', 'abs', 'floor', 'ceil', 'sign')


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def _problems(seed, n, L=48, dtype=np.float32, ops=tl.C1_OPERATORS, Bs=None, Ds=None,
              valid_only=False):
    from warpsymbolic_b200.batch import BatchProblem
    rng = np.random.default_rng(seed)
    out, host = [], []
    for i in range(n):
        V = int(rng.integers(1, 11))
        g = tl.GPUGrammar(num_variables=V, operators=ops)
        B = int(Bs[i]) if Bs is not None else int(rng.integers(1, 700))
        D = int(Ds[i]) if Ds is not None else int(10 ** rng.uniform(1.0, 4.7))
        pop, consts = tl.random_population(g, max(B, 1), L, 4, rng, valid_only=valid_only)
        pop, consts = pop[:B], consts[:B].astype(dtype)
        X = rng.uniform(-4, 4, size=(V, D)).astype(dtype)
        y = (np.sin(X[0]) * 2.0 + X[-1] * X[0]).astype(dtype)
        out.append(BatchProblem(T(pop), T(X), T(y), T(consts), g))
        host.append((g, pop, consts, X, y))
    return out, host


def _single(p, **kw):
    from warpsymbolic_b200.cuda_vm import CudaRPNVM
    vm = CudaRPNVM(p.grammar, DEV)
    nin = torch.empty(p.population.shape[0], dtype=torch.int32, device=DEV)
    out = vm.eval_fitness(p.population, p.x, p.constants, p.y, out_ninvalid=nin, **kw)
    return out.cpu().numpy(), nin.cpu().numpy()


@pytest.mark.parametrize("policy,loss", [("classic", "mse"), ("fused", "rmse"), ("classic", "r2")])
@pytest.mark.parametrize("schedule", [3, 1])
def test_batch_matches_single_problem_calls(policy, loss, schedule):
    from warpsymbolic_b200.batch import BatchedFitness
    Bs = [0, 1, 37, 500, 699, 5, 250, 64, 1, 333, 128, 17]
    Ds = [50, 1, 100, 20000, 3, 700, 45000, 512, 1025, 9999, 2048, 31]
    probs, _ = _problems(7, len(Bs), Bs=Bs, Ds=Ds)
    bf = BatchedFitness(probs, loss=loss, policy=policy, schedule=schedule, count_invalid=True)
    bf.evaluate()
    torch.cuda.synchronize()
    for i, p in enumerate(probs):
        if p.population.shape[0] == 0:
            continue
        want, wn = _single(p, policy=policy, loss=loss, schedule=schedule)
        got, gn = bf.outputs[i].cpu().numpy(), bf.ninvalid[i].cpu().numpy()
        assert np.array_equal(gn, wn), i
        # same schedule, same per-problem chunks and row splits: the same bits
        assert np.array_equal(got, want, equal_nan=True), (i, np.nonzero(got != want)[0][:5])
    bf.close()


def test_batch_f64_exact_operators_match_oracle():
    from warpsymbolic_b200.batch import BatchedFitness
    probs, host = _problems(11, 9, dtype=np.float64, ops=EXACT_OPERATORS)
    bf = BatchedFitness(probs, loss="rmse", policy="classic", count_invalid=True)
    bf.evaluate()
    torch.cuda.synchronize()
    for i, (g, pop, consts, X, y) in enumerate(host):
        ref, rn = tl.oracle_fitness(g, pop, X, consts, y, policy="classic", loss="rmse",
                                    with_ninv=True)
        assert np.array_equal(bf.ninvalid[i].cpu().numpy(), rn)
        tl.assert_fitness_close(bf.outputs[i].cpu().numpy(), ref, rtol=1e-12, atol=1e-300,
                                iv=1e100)


def test_batch_graph_replay_after_in_place_rewrite():
    from warpsymbolic_b200.batch import BatchedFitness
    probs, _ = _problems(5, 6, valid_only=True)
    bf = BatchedFitness(probs, loss="mse", policy="classic")
    g = bf.capture()
    g.replay()
    torch.cuda.synchronize()
    first = [o.clone() for o in bf.outputs]
    # next "generation": every population reversed in place, constants scaled in place
    for p in probs:
        p.population.copy_(torch.flip(p.population, dims=[0]))
        p.constants.mul_(0.5)
    g.replay()
    torch.cuda.synchronize()
    replayed = [o.clone() for o in bf.outputs]
    bf.evaluate()
    torch.cuda.synchronize()
    for a, b, f in zip(replayed, bf.outputs, first):
        assert torch.equal(a, b)
    assert any(not torch.equal(a, f) for a, f in zip(replayed, first))
    del g
    bf.close()


def test_batch_cancel_flag_stops_a_launch_and_the_next_is_exact():
    """A set cancel flag: the evaluator takes no work item and the outputs keep their previous
    values, eagerly and in a graph replay; once the flag is cleared, the next launch (evaluate
    only, on the tapes the cancelled one compiled) and the next replay equal a batch without a
    flag bit for bit, also for problems whose rows are split across CTAs."""
    from warpsymbolic_b200.batch import BatchedFitness
    probs, _ = _problems(9, 5, valid_only=True, Ds=[50_000, 120, 30_000, 8_000, 90_000])
    ref = BatchedFitness(probs, loss="mse", policy="classic")
    ref.evaluate()
    torch.cuda.synchronize()
    want = [o.clone() for o in ref.outputs]
    ref.close()
    bf = BatchedFitness(probs, loss="mse", policy="classic")
    flag = torch.ones(1, dtype=torch.int32, device=DEV)
    bf.set_cancel_flag(flag)
    for o in bf.outputs:
        o.fill_(-7.0)
    bf.evaluate()
    torch.cuda.synchronize()
    assert all(bool((o == -7.0).all()) for o in bf.outputs)
    flag.zero_()
    bf.evaluate(phase=2)
    torch.cuda.synchronize()
    assert all(torch.equal(a, b) for a, b in zip(bf.outputs, want))
    g = bf.capture()
    for o in bf.outputs:
        o.fill_(-7.0)
    flag.fill_(1)
    g.replay()
    torch.cuda.synchronize()
    assert all(bool((o == -7.0).all()) for o in bf.outputs)
    flag.zero_()
    g.replay()
    torch.cuda.synchronize()
    assert all(torch.equal(a, b) for a, b in zip(bf.outputs, want))
    del g
    bf.set_cancel_flag(None)
    bf.close()
    with pytest.raises(ValueError):
        BatchedFitness(probs, loss="mse").set_cancel_flag(torch.ones(2, dtype=torch.int32,
                                                                     device=DEV))


def test_batch_is_independent_of_its_neighbours():
    """A problem's losses do not depend on which other problems share the launch."""
    from warpsymbolic_b200.batch import BatchedFitness
    probs, _ = _problems(9, 8, Bs=[300] * 8, Ds=[40000, 200, 7, 3000, 90, 12345, 1, 640])
    full = BatchedFitness(probs, loss="mse", policy="classic", schedule=3)
    full.evaluate()
    part = BatchedFitness(probs[2:5], loss="mse", policy="classic", schedule=3)
    part.evaluate()
    torch.cuda.synchronize()
    for k in range(3):
        assert torch.equal(full.outputs[2 + k], part.outputs[k])


def test_autotune_picks_a_runnable_schedule():
    from warpsymbolic_b200 import batch
    probs, _ = _problems(3, 5, valid_only=True)
    best, times = batch.autotune(probs, loss="mse", policy="classic", reps=1, use_cache=False)
    assert best in times and times[best] == min(times.values())
    again, t2 = batch.autotune(probs, loss="mse", policy="classic")
    assert again == best and t2 == {}


def test_batch_argument_errors():
    from warpsymbolic_b200.batch import BatchedFitness
    probs, _ = _problems(1, 2, valid_only=True)
    bad = probs[0].__class__(probs[0].population[:, :10].contiguous(), probs[0].x, probs[0].y,
                             probs[0].constants, probs[0].grammar)
    with pytest.raises(RuntimeError, match="population must be uint8"):
        BatchedFitness([probs[1], bad])
