"""Program sharding across GPUs (one process per GPU, torch.distributed).

Programs are independent, so a population is split into contiguous shards, each rank scores its
own shard with the single-GPU evaluator (no collective on the data path), and — only when a
caller needs the whole fitness vector on every rank, for selection over one population spanning
GPUs — the shards are all-gathered ([B] floats: NCCL over NVLink on GPUs, gloo on CPU).  When
requests or problems are sharded instead, no collective is needed at all.

    with ShardedEvaluator(score_fn) as ev:     # inside an initialised process group
        fitness = ev.evaluate(population, ...)  # [B] on every rank

`score_fn(population_shard, constants_shard, *args)` returns the shard's fitness tensor.
"""
from __future__ import annotations

from typing import Callable, Tuple

import torch
import torch.distributed as dist


def shard_bounds(n: int, world: int, rank: int) -> Tuple[int, int]:
    """[start, end) of rank's contiguous shard of n items: sizes differ by at most one, the
    first n % world ranks take the extra item."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d outside world of %d" % (rank, world))
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


class ShardedEvaluator:
    def __init__(self, score_fn: Callable, group=None):
        self.score_fn = score_fn
        self.group = group

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def _world(self):
        if dist.is_available() and dist.is_initialized():
            return dist.get_world_size(self.group), dist.get_rank(self.group)
        return 1, 0

    def evaluate_local(self, population, constants=None, *args, **kw):
        """This rank's shard only: (fitness of the shard, (start, end))."""
        world, rank = self._world()
        s, e = shard_bounds(int(population.shape[0]), world, rank)
        c = constants[s:e] if constants is not None else None
        return self.score_fn(population[s:e], c, *args, **kw), (s, e)

    def evaluate(self, population, constants=None, *args, **kw):
        """The full [B] fitness on every rank (all-gather of the shards)."""
        world, rank = self._world()
        local, _ = self.evaluate_local(population, constants, *args, **kw)
        if world == 1:
            return local
        B = int(population.shape[0])
        sizes = [shard_bounds(B, world, r) for r in range(world)]
        width = max(e - s for s, e in sizes)
        # all_gather wants equal shapes: pad every shard to the widest one
        buf = torch.zeros(width, dtype=local.dtype, device=local.device)
        buf[:local.numel()] = local
        parts = [torch.empty_like(buf) for _ in range(world)]
        dist.all_gather(parts, buf, group=self.group)
        return torch.cat([p[:e - s] for p, (s, e) in zip(parts, sizes)])


def max_over_ranks(seconds: float, device=None) -> float:
    """The largest of every rank's timing (the multi-GPU time of a step)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return seconds
    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
