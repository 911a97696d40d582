"""Program and row sharding across GPUs (one process per GPU, torch.distributed).

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

from typing import Callable, Optional, Tuple

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


class RowShardedEvaluator:
    """One population scored on a data set whose ROWS are split across ranks (a data set too
    large for one GPU, or D >= 10^6): every rank scores all programs on its contiguous row shard
    -- per-program sum of squared errors (FP64) and invalid-row count, the classic-path partial
    sums -- the partials and the shard's (n, sum y, sum y^2) are summed over ranks in one
    all-reduce, and every rank forms the same loss with the evaluator's rules (`combine`).

        ev = RowShardedEvaluator(vm)                       # vm: CudaRPNVM of the grammar
        loss = ev.evaluate(population, x_shard, y_shard, constants, loss="rmse")

    `partial_fn(population, x_shard, y_shard, constants) -> (sse float64 [B], ninv int [B])`
    replaces the GPU evaluator (the CPU tests pass the oracle).  The classic policy only: its
    program-level rules need the sums alone, while the fused policy also flags per-row
    overflow.  Results agree with a single-GPU evaluation up to the order of the FP64 sums."""

    def __init__(self, vm=None, group=None, strict_mode: int = 0,
                 invalid_value: Optional[float] = None, partial_fn: Optional[Callable] = None):
        self.vm = vm
        self.group = group
        self.strict_mode = int(strict_mode)
        self.invalid_value = invalid_value
        self.partial_fn = partial_fn

    def _world(self):
        if dist.is_available() and dist.is_initialized():
            return dist.get_world_size(self.group), dist.get_rank(self.group)
        return 1, 0

    def partial(self, population, x_shard, y_shard, constants=None):
        """(sse float64 [B], invalid-row count [B]) of this rank's rows."""
        if self.partial_fn is not None:
            return self.partial_fn(population, x_shard, y_shard, constants)
        B = int(population.shape[0])
        ninv = torch.empty(B, dtype=torch.int32, device=x_shard.device)
        sse = self.vm.eval_fitness(population, x_shard, constants, y_shard,
                                   strict_mode=self.strict_mode, policy="classic", loss="sse",
                                   out_ninvalid=ninv, invalid_value=0.0)
        return sse, ninv

    @staticmethod
    def pack(sse, ninv, y_shard) -> torch.Tensor:
        """[2B + 3] float64: the partial sums and the shard's (n, sum y, sum y^2)."""
        y = y_shard.reshape(-1).to(torch.float64)
        stats = torch.stack([torch.tensor(float(y.numel()), dtype=torch.float64,
                                          device=y.device), y.sum(), (y * y).sum()])
        return torch.cat([sse.to(torch.float64).reshape(-1),
                          ninv.to(torch.float64).reshape(-1).to(sse.device), stats.to(sse.device)])

    @staticmethod
    def combine(total: torch.Tensor, B: int, dtype, loss: str = "mse",
                invalid_value: Optional[float] = None) -> torch.Tensor:
        """Losses [B] (dtype) from the summed pack: the evaluator's final rules -- an invalid row
        makes the program invalid (invalid_value; its negative for R^2), an overflowing sum
        gives sqrt(invalid_value) for RMSE, else MSE = SSE / D rounded to dtype, RMSE its square
        root, R^2 = 1 - MSE / Var(y)."""
        if invalid_value is None:
            invalid_value = 1e15 if dtype == torch.float32 else 1e100
        sse, ninv, (n, sy, syy) = total[:B], total[B:2 * B], total[2 * B:2 * B + 3]
        tmax = torch.finfo(dtype).max
        iv = float(invalid_value)
        invalid = ninv > 0
        ovf = ~(sse <= tmax)
        mse = sse / n
        mse_t = mse.to(dtype)
        if loss == "mse":
            good = mse_t.to(torch.float64)
            bad_inv, bad_ovf = iv, iv
        elif loss == "rmse":
            q = torch.sqrt(mse_t)
            good = torch.where(torch.isfinite(q), q.to(torch.float64),
                               torch.full_like(mse, iv))
            bad_inv = iv
            bad_ovf = float(torch.sqrt(torch.tensor(iv, dtype=dtype)))
        elif loss == "r2":
            mean = sy / n
            yvar = syy / n - mean * mean
            if float(yvar) > 0.0:
                good = 1.0 - mse / yvar
            else:
                good = torch.where(mse == 0.0, torch.ones_like(mse), torch.full_like(mse, -iv))
            bad_inv, bad_ovf = -iv, -iv
        else:
            raise ValueError("loss must be mse, rmse or r2")
        out = torch.where(invalid, torch.full_like(mse, bad_inv),
                          torch.where(ovf, torch.full_like(mse, bad_ovf), good))
        return out.to(dtype)

    def evaluate(self, population, x_shard, y_shard, constants=None, loss: str = "mse"):
        """The loss [B] of every program over all ranks' rows, on every rank."""
        world, _ = self._world()
        sse, ninv = self.partial(population, x_shard, y_shard, constants)
        total = self.pack(sse, ninv, y_shard)
        if world > 1:
            dist.all_reduce(total, op=dist.ReduceOp.SUM, group=self.group)
        return self.combine(total, int(population.shape[0]), x_shard.dtype, loss,
                            self.invalid_value)
