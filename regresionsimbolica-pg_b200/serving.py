"""A serving loop for fit and evaluate requests with continuous batching.

Requests of different sizes arrive over time.  Each admitted request keeps its state on the
device (data set, population, constants, losses) until it completes.  Admitted requests are
grouped by the work of one of their generations (programs x rows, in doublings); a step of a
group is ONE batched evaluation of its requests (libwarpsym's ws_batch_*) and ONE batched GP
generation for its fits that still have generations to run (ws_gp_*).  A tick steps every group,
the cheaper groups several times (2^j times for j doublings below the most expensive, up to 8),
so small fits are not held to the pace of the large ones they share the GPU with.  Requests
that arrive while a tick runs are admitted at the next tick, in arrival order, as long as their
estimated device footprint fits the memory budget and a slot is free.

    server = ContinuousBatchingServer(hbm_budget=8 << 30)
    results = server.serve(requests)           # Result per request: latency, losses, best program

  evaluate request: the losses of its programs on its data set (one tick);
  fit request: `generations` rounds of evaluate + breed, then a final evaluation; the result is
    the best program of the last population with its constants and loss.

A request's result does not depend on what else is served with it: a problem's losses are
bit-identical whatever shares the launch (same schedule), and its offspring depend only on its
own seed, generation count, population and losses.  `serve_plain` is the one-request-at-a-time
path (each request alone, one launch sequence per evaluation and per generation) on the same
stream, for comparison.
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np
import torch

from .batch import BatchProblem, BatchedFitness
from .gp import GPStep


@dataclass
class Request:
    rid: int
    kind: str                   # "fit" or "evaluate"
    grammar: object             # GPUGrammar (variables and operators of this request)
    X: np.ndarray               # [V, D] float32
    y: np.ndarray               # [D] float32
    population: np.ndarray      # [B, L] uint8: programs to score, or the initial population
    constants: np.ndarray       # [B, K] float32
    generations: int = 0        # fit: generations to breed
    seed: int = 0               # fit: random stream of the GP step
    arrival: float = 0.0        # seconds after the start of the stream


@dataclass
class Result:
    rid: int
    kind: str
    arrival: float
    admitted: float
    done: float
    losses: Optional[np.ndarray] = None          # evaluate: [B]
    best_loss: Optional[float] = None            # fit
    best_program: Optional[np.ndarray] = None    # fit: [L] uint8
    best_constants: Optional[np.ndarray] = None  # fit: [K]
    generations: int = 0

    @property
    def latency(self) -> float:
        return self.done - self.arrival


@dataclass
class _Group:
    """Admitted requests of one cost class with the plans that serve them together."""
    slots: list = field(default_factory=list)
    key: Optional[tuple] = None
    bf: Optional[BatchedFitness] = None
    gp: Optional[GPStep] = None
    breeders: list = field(default_factory=list)


@dataclass
class _Slot:
    req: Request
    prob: BatchProblem
    nbytes: int
    admitted: float
    gen: int = 0


class _Pool:
    """One device buffer reused by every plan of a serving run (plans change with the batch
    membership; work on one stream is ordered, so a new plan may take over the memory that
    queued ticks of the previous plan still use).  It grows by at least half when a plan needs
    more; a replaced buffer is kept until the ticks queued before the growth have finished."""

    def __init__(self, device):
        self.device = device
        self.buf: Optional[torch.Tensor] = None
        self.retired: List[torch.Tensor] = []

    def __call__(self, nbytes: int) -> torch.Tensor:
        if self.buf is None or self.buf.numel() < nbytes:
            if self.buf is not None:
                self.retired.append(self.buf)
            grow = 0 if self.buf is None else self.buf.numel() * 3 // 2
            self.buf = torch.empty(max(int(nbytes), grow), dtype=torch.uint8, device=self.device)
        return self.buf


def footprint(req: Request, L: Optional[int] = None) -> int:
    """Estimated device bytes of an admitted request: data set, population, constants and
    losses, the evaluator's per-program scratch (header, tape, order, partial sums) and the GP
    step's scratch generation."""
    B, L = req.population.shape if L is None else (req.population.shape[0], L)
    K = req.constants.shape[1] if req.constants.ndim == 2 else 0
    V, D = req.X.shape
    data = 4 * (V + 1) * D
    per_prog = L + 4 * K + 4 + 16 + 8 * L + 4 + 8 + 4 + 16 * 8
    gp = (L + 4 * K) if req.kind == "fit" else 0
    return int(data + B * (per_prog + gp) + (1 << 20))


class ContinuousBatchingServer:
    def __init__(self, device=None, hbm_budget: Optional[int] = None, max_active: int = 64,
                 schedule: int = 3, loss: str = "mse", gp_options: Optional[Dict] = None):
        self.device = torch.device(device) if device is not None else torch.device("cuda", 0)
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            hbm_budget = int(free * 0.5)
        self.hbm_budget = int(hbm_budget)
        self.max_active = int(max_active)
        self.schedule = int(schedule)
        self.loss = loss
        self.gp_options = dict(gp_options or {})
        self.stats: Dict[str, float] = {}

    def _admit(self, req: Request, now: float) -> _Slot:
        d = self.device
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(d)
        prob = BatchProblem(t(req.population.astype(np.uint8)), t(req.X.astype(np.float32)),
                            t(req.y.astype(np.float32)), t(req.constants.astype(np.float32)),
                            req.grammar)
        return _Slot(req, prob, footprint(req), now)

    @staticmethod
    def cost_class(req: Request) -> int:
        """Work class of one generation of a request: doublings of programs x rows."""
        work = max(1, int(req.population.shape[0]) * int(req.X.shape[1]))
        return max(0, int(np.log2(work)))

    def serve(self, requests: Sequence[Request], realtime: bool = True,
              max_inflight: int = 8, max_steps_per_tick: int = 8) -> List[Result]:
        """Serves the stream; with realtime=False arrivals only order the queue (a request is
        admitted as soon as it is first in line and fits).

        Admitted requests are grouped by the work of one of their generations (cost_class);
        each group has its own batch plan and GP step, replanned only when its membership
        changes.  A tick runs every group once, and a group that is 2^j times cheaper than the
        most expensive one runs min(2^j, max_steps_per_tick) generations in that tick, so a small
        fit does not wait for the large fits it shares the GPU with.  Steps are queued on the
        GPU without waiting for each other; at most `max_inflight` steps are in flight.  Results
        are read back (pinned memory) when the step that finishes them completes; completion
        times come from CUDA events.  A request stays in its group for life: its losses and
        offspring are the same whatever it is served with."""
        reqs = sorted(requests, key=lambda r: (r.arrival, r.rid))
        waiting: collections.deque = collections.deque()
        groups: Dict[int, _Group] = {}
        results: List[Result] = []
        inflight: collections.deque = collections.deque()  # (event, [(slot, host losses, snap)])
        used = 0
        i = 0
        steps = max_active_seen = 0
        stream = torch.cuda.current_stream(self.device)
        torch.cuda.synchronize(self.device)
        t0 = time.perf_counter()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        retired = []  # plans still referenced by queued work
        pools = {}

        def drain_one():
            nonlocal used
            ev, items = inflight.popleft()
            ev.synchronize()
            done_t = ev0.elapsed_time(ev) / 1e3
            for slot, hl, snap in items:
                r = slot.req
                res = Result(r.rid, r.kind, r.arrival, slot.admitted, done_t)
                losses = hl.numpy()
                if r.kind == "evaluate":
                    res.losses = losses.copy()
                else:
                    b = int(np.argmin(np.where(np.isnan(losses), np.inf, losses)))
                    pop, cst = snap
                    res.best_loss = float(losses[b])
                    res.best_program = pop[b].numpy().copy()
                    res.best_constants = cst[b].numpy().copy()
                    res.generations = slot.gen
                results.append(res)
                used -= slot.nbytes

        def step(cls: int, grp: "_Group") -> None:
            """One generation of a group: evaluate everything, read back what finishes, breed
            the rest."""
            nonlocal steps
            active = grp.slots
            breed = [s for s in active if s.req.kind == "fit" and s.gen < s.req.generations]
            k = (tuple(s.req.rid for s in active), tuple(s.req.rid for s in breed))
            if k != grp.key:  # membership changed: plan the group again (stream-ordered)
                retired.extend(x for x in (grp.gp, grp.bf) if x is not None)
                if cls not in pools:
                    pools[cls] = (_Pool(self.device), _Pool(self.device))
                ep, gpp = pools[cls]
                grp.bf = BatchedFitness([s.prob for s in active], loss=self.loss,
                                        policy="classic", schedule=self.schedule, workspace=ep)
                grp.gp = None
                grp.breeders = breed
                if breed:
                    idx = {s.req.rid: j for j, s in enumerate(active)}
                    grp.gp = GPStep([s.prob for s in breed],
                                    [grp.bf.outputs[idx[s.req.rid]] for s in breed],
                                    [s.req.seed for s in breed],
                                    generations=[s.gen for s in breed], workspace=gpp,
                                    **self.gp_options)
                grp.key = k
            bf = grp.bf
            bf.evaluate()
            finished = [s for s in active if s.req.kind == "evaluate" or s.gen >= s.req.generations]
            items = []
            for j, s in enumerate(active):
                if s in finished:
                    hl = torch.empty(bf.outputs[j].numel(), dtype=bf.outputs[j].dtype,
                                     pin_memory=True)
                    hl.copy_(bf.outputs[j], non_blocking=True)
                    snap = None
                    if s.req.kind == "fit":
                        snap = (torch.empty(s.prob.population.shape, dtype=torch.uint8,
                                            pin_memory=True),
                                torch.empty(s.prob.constants.shape, dtype=s.prob.constants.dtype,
                                            pin_memory=True))
                        snap[0].copy_(s.prob.population, non_blocking=True)
                        snap[1].copy_(s.prob.constants, non_blocking=True)
                    items.append((s, hl, snap))
            if grp.gp is not None:
                grp.gp.step()
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(stream)
            inflight.append((ev, items))
            steps += 1
            for s in grp.breeders:
                s.gen += 1
            if finished:
                gone = {s.req.rid for s in finished}
                grp.slots = [s for s in active if s.req.rid not in gone]
            while len(inflight) > max_inflight:
                drain_one()

        while i < len(reqs) or waiting or any(g.slots for g in groups.values()) or inflight:
            now = time.perf_counter() - t0
            while i < len(reqs) and (reqs[i].arrival <= now or not realtime):
                waiting.append(reqs[i])
                i += 1
            n_active = sum(len(g.slots) for g in groups.values())
            while (waiting and n_active < self.max_active
                   and (n_active == 0 or used + footprint(waiting[0]) <= self.hbm_budget)):
                r = waiting.popleft()
                s = self._admit(r, max(now, r.arrival) if realtime else now)
                used += s.nbytes
                groups.setdefault(self.cost_class(r), _Group()).slots.append(s)
                n_active += 1
            if n_active == 0:
                if inflight:
                    drain_one()
                elif i < len(reqs) and realtime:
                    time.sleep(max(0.0, reqs[i].arrival - (time.perf_counter() - t0)))
                continue
            max_active_seen = max(max_active_seen, n_active)
            live = sorted(c for c, g in groups.items() if g.slots)
            top = live[-1]
            for cls in live:  # cheapest first: the quickest requests finish soonest
                grp = groups[cls]
                reps = min(max_steps_per_tick, 1 << min(top - cls, 30))
                for _ in range(reps):
                    if not grp.slots:
                        break
                    step(cls, grp)
            if not inflight:
                if len(retired) > 8:
                    retired.clear()
                for ep, gpp in pools.values():
                    ep.retired.clear()
                    gpp.retired.clear()
        while inflight:
            drain_one()
        torch.cuda.synchronize(self.device)
        for g in groups.values():
            retired.extend(x for x in (g.gp, g.bf) if x is not None)
        for x in retired:
            x.close()
        self.stats = {"ticks": steps, "max_active": max_active_seen,
                      "groups": len(groups), "makespan_s": time.perf_counter() - t0}
        return sorted(results, key=lambda r: r.rid)


def serve_plain(requests: Sequence[Request], device=None, schedule: int = 3, loss: str = "mse",
                gp_options: Optional[Dict] = None, realtime: bool = True) -> List[Result]:
    """One request at a time in arrival order, each with its own launches: one evaluation launch
    sequence (ws_eval_fitness) per evaluation and one GP step per generation."""
    from .cuda_vm import CudaRPNVM
    dev = torch.device(device) if device is not None else torch.device("cuda", 0)
    results = []
    t0 = time.perf_counter()
    for r in sorted(requests, key=lambda q: (q.arrival, q.rid)):
        if realtime:
            time.sleep(max(0.0, r.arrival - (time.perf_counter() - t0)))
        admitted = time.perf_counter() - t0
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        prob = BatchProblem(t(r.population.astype(np.uint8)), t(r.X.astype(np.float32)),
                            t(r.y.astype(np.float32)), t(r.constants.astype(np.float32)), r.grammar)
        vm = CudaRPNVM(r.grammar, dev)
        out = torch.empty(prob.population.shape[0], dtype=torch.float32, device=dev)

        def evaluate():
            vm.eval_fitness(prob.population, prob.x, prob.constants, prob.y, policy="classic",
                            loss=loss, out=out, schedule=schedule)
        res = Result(r.rid, r.kind, r.arrival, admitted, 0.0)
        if r.kind == "evaluate":
            evaluate()
            res.losses = out.cpu().numpy()
        else:
            gp = GPStep([prob], [out], [r.seed], **(gp_options or {}))
            for _ in range(r.generations):
                evaluate()
                gp.step()
            evaluate()
            losses = out.cpu().numpy()
            b = int(np.argmin(np.where(np.isnan(losses), np.inf, losses)))
            res.best_loss = float(losses[b])
            res.best_program = prob.population[b].cpu().numpy()
            res.best_constants = prob.constants[b].cpu().numpy()
            res.generations = r.generations
            gp.close()
        torch.cuda.synchronize(dev)
        res.done = time.perf_counter() - t0
        results.append(res)
    return sorted(results, key=lambda q: q.rid)


def latency_summary(results: Sequence[Result], makespan: float) -> Dict[str, float]:
    lat = np.array([r.latency for r in results])
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "requests": len(results),
            "throughput_req_s": len(results) / makespan if makespan > 0 else 0.0}
