"""Structural hashing and deduplication exports against the reference extension's kernels and a
numpy restatement: hashes and variable masks bit for bit, sharing penalties bit for bit, dedup
groups and counts equal (the original of a group is the lowest index here; the reference picks
by thread timing), replacement positions the same set (ascending here)."""
import numpy as np
import pytest
import torch

import refext
import ws_testlib as tl

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(refext.path("fastmath") is None,
                               reason="reference extension not built (oracle/build_ref.sh)")
DEV = torch.device("cuda:0") if torch.cuda.is_available() else None


def _pop(B=6000, L=32, dup_frac=0.4, seed=0):
    rng = np.random.default_rng(seed)
    g = tl.GPUGrammar(num_variables=6, operators=tl.C1_OPERATORS)
    pop = tl.synthetic.random_programs(g, B, 1, 12, L, rng, max_consts=3)
    idx = rng.integers(0, B, size=int(B * dup_frac))
    pop[rng.integers(0, B, size=len(idx))] = pop[idx]   # planted duplicates
    return g, pop


def _np_hash(pop, pad=0):
    h = np.zeros(len(pop), dtype=np.uint64)
    for b, row in enumerate(pop):
        acc, p = np.uint64(0), np.uint64(1)
        for t in row:
            if t == pad:
                break
            acc = acc + np.uint64(t) * p
            p = p * np.uint64(31)
        h[b] = acc
    return h.view(np.int64)


def test_hashes_and_presence():
    from warpsymbolic_b200 import rpn_cuda_native as ours
    g, pop = _pop(B=800)
    x0 = g.token_to_id["x0"]
    h = torch.empty(len(pop), dtype=torch.int64, device=DEV)
    vp = torch.empty(len(pop), dtype=torch.int32, device=DEV)
    with np.errstate(over="ignore"):
        ours.compute_population_hashes(torch.from_numpy(pop).to(DEV), h, vp, 0, x0, 6)
        assert np.array_equal(h.cpu().numpy(), _np_hash(pop))
    want = np.array([sum(1 << (t - x0) for t in set(r[:np.argmax(r == 0) if (r == 0).any() else len(r)])
                         if x0 <= t < x0 + 6) for r in pop], dtype=np.int32)
    assert np.array_equal(vp.cpu().numpy(), want)
    vp2 = torch.zeros_like(vp)
    ours.compute_var_presence(torch.from_numpy(pop).to(DEV), vp2, 0, x0, 6)
    assert torch.equal(vp, vp2)


@needs_ref
def test_identical_to_reference():
    from warpsymbolic_b200 import rpn_cuda_native as ours
    ref = refext.load("fastmath")
    g, pop = _pop()
    P = torch.from_numpy(pop).to(DEV)
    x0 = g.token_to_id["x0"]
    res = {}
    for name, mod in (("ref", ref), ("ours", ours)):
        h = torch.empty(len(pop), dtype=torch.int64, device=DEV)
        vp = torch.empty(len(pop), dtype=torch.int32, device=DEV)
        mod.compute_population_hashes(P, h, vp, 0, x0, 6)
        table = torch.full((1 << 20,), -1, dtype=torch.int64, device=DEV)
        dup = torch.empty(len(pop), dtype=torch.int32, device=DEV)
        orig = torch.empty(len(pop), dtype=torch.int64, device=DEV)
        mod.structural_dedup(h, table, dup, orig)
        n_u = mod.count_unique(dup)
        pos = torch.empty(len(pop), dtype=torch.int64, device=DEV)
        nr = torch.zeros(1, dtype=torch.int64, device=DEV)
        n_r = mod.get_replacement_positions(dup, pos, nr)
        pen = mod.fitness_sharing_penalty(P, 3, 2000, 2, 8)
        res[name] = dict(h=h.cpu().numpy(), vp=vp.cpu().numpy(), dup=dup.cpu().numpy(),
                         orig=orig.cpu().numpy(), n_u=n_u, n_r=n_r,
                         pos=np.sort(pos.cpu().numpy()[:n_r]), pen=pen.cpu().numpy())
    r, o = res["ref"], res["ours"]
    for k in ("h", "vp", "pen"):
        assert np.array_equal(r[k], o[k]), k
    assert r["n_u"] == o["n_u"] == len(np.unique(o["h"]))
    assert r["n_r"] == o["n_r"] == len(pop) - o["n_u"]
    # same groups: equal hashes <=> same original; ours is the lowest index of its group
    for d in (r, o):
        assert np.array_equal(d["h"][d["orig"]], d["h"])
        assert (d["dup"] == (d["orig"] != np.arange(len(pop)))).all()
    first = {}
    for i, hv in enumerate(o["h"]):
        first.setdefault(hv, i)
    assert np.array_equal(o["orig"], np.array([first[hv] for hv in o["h"]]))
    # each side lists exactly its own duplicate flags (which member of a group is flagged
    # differs: the reference keeps whichever thread claimed the slot first)
    for d in (r, o):
        assert np.array_equal(d["pos"], np.nonzero(d["dup"])[0])
    assert (o["pen"] > 0).any()


@pytest.mark.parametrize("B,shift", [(100_003, 0), (70_001, 1), (16_384, 0), (16_385, 1),
                                     (1, 0), (0, 0)])
def test_replacement_positions_and_count_across_tiles(B, shift):
    """The flag scan walks tiles of 16,384 flags: several tiles, a partial last tile, and a
    flag array whose base is not 16-byte aligned (scalar loads) against numpy."""
    from warpsymbolic_b200 import rpn_cuda_native as ours
    rng = np.random.default_rng(B + shift)
    flags = (rng.random(B) < 0.3).astype(np.int32)
    buf = torch.empty(B + 4, dtype=torch.int32, device=DEV)
    dup = buf[shift:shift + B]
    dup.copy_(torch.from_numpy(flags).to(DEV))
    assert ours.count_unique(dup) == int((flags == 0).sum())
    pos = torch.empty(max(B, 1), dtype=torch.int64, device=DEV)
    nr = torch.zeros(1, dtype=torch.int64, device=DEV)
    n = ours.get_replacement_positions(dup, pos, nr)
    want = np.nonzero(flags == 1)[0]
    assert n == len(want) == int(nr.item())
    assert np.array_equal(pos.cpu().numpy()[:n], want)
