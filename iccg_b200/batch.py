"""Many independent solves on one GPU: batched systems and a serving loop.

A system lives in a context: the system's matrix, schedule, IC(0) factor
and lane-interleaved layout resident in device memory.  The batched engine
(``iccg_b200.Batch``, the iccg_batch C ABI) advances many solves together,
every CG kernel one launch over all of them; a solve's arithmetic does not
depend on what else runs, so each result is the same bits alone and in the
mix.

* ``ServingLoop`` takes requests as they arrive (continuous batching): it
  admits them by free device memory, builds their systems on builder
  threads, submits each into a slot of one batch session, steps all running
  solves together and retires the stopped ones between steps.  It reports
  p50 / p99 latency (arrival to result) and solves/s.
* ``solve_batch`` and ``ThreadedServingLoop`` are the earlier forms, one
  context and CUDA stream per system driven by host threads; they remain as
  the comparisons.
"""
from __future__ import annotations

import queue as _queue
import statistics
import threading
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence

import numpy as np

from . import OPT_STAGE_ROWS, STORE_FP32, STORE_FP64, MODE_FUSED, PRECOND_IC0, Batch, Context, device_memory
from .problems import Problem


@dataclass
class SolveRecord:
    system: int
    rhs: int
    iters: int
    converged: bool
    true_rel_resid: float
    device_ms: float       # the solve's device time (CUDA events)
    wall_ms: float         # host time of the call, copies included
    x: Optional[np.ndarray] = None


class ResidentSystem:
    """One system on the device: A_run, schedule and IC(0) factor resident.

    With `ctx` the system is loaded into that (borrowed) context, replacing
    whatever it held; the context's device buffers are reused where they are
    large enough, and close() leaves the context open."""

    def __init__(self, P: Problem, device: int = 0, storage: int = STORE_FP32, ctx: Optional[Context] = None):
        self.P = P
        self.storage = storage
        self._own = ctx is None
        self.ctx = Context(device) if ctx is None else ctx
        self.ctx.upload(P.A_run)
        self.ctx.set_schedule(P.sched)
        self.ctx.build(P.precond_kind if P.precond_kind != 2 else PRECOND_IC0, 0.0)

    @property
    def device_bytes(self) -> int:
        return self.ctx.device_bytes

    def solve(self, b_run: np.ndarray, tol: float = 1e-8, max_iter: int = 10000, mode: int = MODE_FUSED,
              rr_interval: int = 50):
        x = np.zeros(self.P.A_run.n)
        t0 = time.perf_counter()
        res = self.ctx.solve(b_run, x, max_iter, tol, mode=mode, storage=self.storage, rr_interval=rr_interval)
        return x, res, (time.perf_counter() - t0) * 1e3

    def close(self):
        if self._own:
            self.ctx.close()


def solve_batch(systems: Sequence[ResidentSystem], rhs: Sequence[Sequence[np.ndarray]], threads: int = 8,
                tol: float = 1e-8, keep_x: bool = False) -> List[SolveRecord]:
    """Solves rhs[i][j] on systems[i] for every i, j; system i's right-hand
    sides run in order on one thread, the systems on `threads` threads."""

    def work(i: int) -> List[SolveRecord]:
        out = []
        for j, b in enumerate(rhs[i]):
            x, res, wall = systems[i].solve(b, tol)
            out.append(SolveRecord(i, j, res.iters, res.converged, res.true_rel_resid, res.solve_ms, wall,
                                   x if keep_x else None))
        return out

    with ThreadPoolExecutor(max_workers=max(1, threads)) as ex:
        parts = list(ex.map(work, range(len(systems))))
    return [r for p in parts for r in p]


def percentile(v: Sequence[float], q: float) -> float:
    if not v:
        return 0.0
    return float(np.percentile(np.asarray(v, dtype=np.float64), q))


@dataclass
class Request:
    rid: int
    arrival_s: float                     # seconds after the loop starts
    build: Callable[[], Problem]         # makes the system (host set-up) when admitted
    est_bytes: int                       # device memory it will hold (admission)


@dataclass
class ServingStats:
    latencies_ms: List[float] = field(default_factory=list)
    iters: List[int] = field(default_factory=list)
    service_ms: List[float] = field(default_factory=list)   # device time admission -> stop
    failed: int = 0
    errors: List[str] = field(default_factory=list)          # why each failed request failed
    elapsed_s: float = 0.0
    peak_bytes: int = 0
    max_in_flight: int = 0

    def fail(self, rid: int, why: str):
        self.failed += 1
        self.errors.append(f"request {rid}: {why}")

    def summary(self) -> dict:
        n = len(self.latencies_ms)
        out = {"solves": n, "failed": self.failed, "elapsed_s": round(self.elapsed_s, 3),
               "solves_per_s": round(n / self.elapsed_s, 3) if self.elapsed_s > 0 else 0.0,
               "p50_ms": round(percentile(self.latencies_ms, 50), 3),
               "p99_ms": round(percentile(self.latencies_ms, 99), 3),
               "mean_iters": round(statistics.mean(self.iters), 1) if self.iters else 0.0,
               "peak_device_bytes": self.peak_bytes}
        if self.service_ms:
            out["device_service_ms"] = {"p50": round(percentile(self.service_ms, 50), 3),
                                        "p99": round(percentile(self.service_ms, 99), 3)}
        if self.max_in_flight:
            out["max_solves_in_flight"] = self.max_in_flight
        if self.errors:
            out["errors"] = self.errors[:5]
        return out


class ThreadedServingLoop:
    """Independent solves on worker threads, one context each (the form the
    continuous-batching ServingLoop replaces; kept as its comparison).

    Requests are admitted in arrival order once they have arrived, as long as
    the admitted solves' device memory stays within `budget_bytes` and a
    worker slot is free. An admitted request builds its system (host set-up,
    upload, IC(0) on the device) and solves it. Up to `workers` solves
    overlap on the GPU.

    With `pool` (the default) each worker keeps one context for the whole
    run: a request loads its system into a free worker context, whose device
    buffers only grow, so a steady stream of requests neither allocates nor
    frees device memory (cudaFree would synchronise the whole device and
    stall the other solves in flight). Without it every request creates and
    destroys its own context. The pooled contexts hold at most `workers`
    times the largest system served.
    """

    def __init__(self, budget_bytes: int, workers: int = 8, device: int = 0, storage: int = STORE_FP32,
                 tol: float = 1e-8, pool: bool = True,
                 make_system: Callable = None, make_context: Callable = None):
        self.budget = budget_bytes
        self.workers = workers
        self.device = device
        self.storage = storage
        self.tol = tol
        self.pool = pool
        # system(P, device, storage, ctx) and context(device) factories:
        # ResidentSystem and Context (tests substitute stand-ins)
        self.make_system = make_system or ResidentSystem
        self.make_context = make_context or Context

    def run(self, requests: Sequence[Request]) -> ServingStats:
        stats = ServingStats()
        lock = threading.Condition()
        in_use = [0]
        queue = sorted(requests, key=lambda r: r.arrival_s)
        t_start = time.perf_counter()

        free_ctx: List[Context] = []
        all_ctx: List[Context] = []
        held_by: dict = {}  # id(pooled context) -> its device bytes, recorded by the worker using it

        def serve(req: Request):
            ctx = None
            try:
                P = req.build()
                if self.pool:
                    with lock:
                        ctx = free_ctx.pop() if free_ctx else None
                    if ctx is None:
                        # a new worker context, created outside the lock
                        ctx = self.make_context(self.device)
                        with lock:
                            all_ctx.append(ctx)
                sysm = self.make_system(P, self.device, self.storage, ctx=ctx)
                try:
                    mine = sysm.device_bytes  # read by the thread that uses the context
                    with lock:
                        if self.pool:
                            held_by[id(ctx)] = mine
                            held = sum(held_by.values())
                        else:
                            held = in_use[0] - req.est_bytes + mine
                        stats.peak_bytes = max(stats.peak_bytes, held)
                    _, res, _ = sysm.solve(P.b_run, self.tol)
                finally:
                    sysm.close()
                done = time.perf_counter() - t_start
                with lock:
                    if res.converged:
                        stats.latencies_ms.append((done - req.arrival_s) * 1e3)
                        stats.iters.append(res.iters)
                    else:
                        stats.fail(req.rid, f"not converged after {res.iters} iterations")
            except Exception as e:
                with lock:
                    stats.fail(req.rid, repr(e))
            finally:
                with lock:
                    if ctx is not None:
                        free_ctx.append(ctx)
                    in_use[0] -= req.est_bytes
                    lock.notify_all()

        with ThreadPoolExecutor(max_workers=max(1, self.workers)) as ex:
            active = []
            for req in queue:
                # wait for the arrival time
                delay = req.arrival_s - (time.perf_counter() - t_start)
                if delay > 0:
                    time.sleep(delay)
                with lock:
                    # admission: memory budget and a free worker
                    while in_use[0] + req.est_bytes > self.budget and in_use[0] > 0:
                        lock.wait(timeout=1.0)
                    while sum(1 for f in active if not f.done()) >= self.workers:
                        lock.wait(timeout=0.05)
                    in_use[0] += req.est_bytes
                active.append(ex.submit(serve, req))
            for f in active:
                f.result()
        stats.elapsed_s = time.perf_counter() - t_start
        for c in all_ctx:
            c.close()
        return stats


# Staged-batch row cap of the contexts behind the batched engine: its work
# lists take each staged batch as one item, and 512 rows (256 is the
# single-system default) gave 1 888 against 1 508 solves/s on 128 systems x 4
# right-hand sides of the batched workload (1 024 and 2 048: no change).
BATCH_STAGE_ROWS = 512


def batch_context(device: int = 0) -> Context:
    """A context for a system that will run on the batched engine."""
    ctx = Context(device)
    ctx.set_option(OPT_STAGE_ROWS, BATCH_STAGE_ROWS)
    return ctx


def load_system(ctx: Context, P: Problem, storage: int):
    """A request's system into a (pooled) context: A_run, schedule, IC(0) on
    the device, and the lane-interleaved layout for `storage`."""
    ctx.upload(P.A_run)
    ctx.set_schedule(P.sched)
    ctx.build(PRECOND_IC0, 0.0)
    ctx.sweep_plan(storage)


class ServingLoop:
    """Continuous batching of independent solves on the batched engine.

    Requests are taken in arrival order once they have arrived.  A request is
    admitted when its estimated device memory fits the free device memory
    (cudaMemGetInfo, plus what idle pooled contexts hold, minus `reserve_bytes`
    and what admitted systems still being built will allocate) and the
    admitted total stays within `budget_bytes`.  Builder threads make each
    admitted system (host set-up, upload, IC(0) and the sweep layout on the
    device) in a context from a pool.  The stepping thread (the caller's)
    then adds the system to one Batch session and submits the solve into a
    slot; every step advances all running solves `graph_iters` iterations in
    one graph launch, and the solves that stopped are retired (solution back
    to the host, slot and context freed) before the next step admits more.
    Each result is the same bits as the solve alone (the batched engine's
    guarantee).  Latency is arrival to retirement.

    make_batch / make_context / load / free_memory default to the device
    (Batch, Context, load_system, cudaMemGetInfo); tests substitute stand-ins.
    """

    def __init__(self, budget_bytes: int, device: int = 0, storage: int = STORE_FP32, tol: float = 1e-8,
                 slots: int = 1024, builders: int = 8, reserve_bytes: int = 2 << 30, graph_iters: int = 4,
                 max_iter: int = 10000, rr_interval: int = 50, make_batch: Callable = None,
                 make_context: Callable = None, load: Callable = None, free_memory: Callable = None):
        self.budget = budget_bytes
        self.device = device
        self.storage = storage
        self.tol = tol
        self.slots = slots
        self.builders = max(1, builders)
        self.reserve = reserve_bytes
        self.graph_iters = graph_iters
        self.max_iter = max_iter
        self.rr_interval = rr_interval
        self.make_batch = make_batch or Batch
        self.make_context = make_context or batch_context
        self.load = load or load_system
        self.free_memory = free_memory or (lambda dev: device_memory(dev)[0])

    def _build(self, req: Request, ctx, ready: "_queue.Queue"):
        try:
            P = req.build()
            if ctx is None:
                ctx = self.make_context(self.device)
            self.load(ctx, P, self.storage)
            ready.put((req, ctx, P, None))
        except Exception as e:  # reported with the request, never dropped
            ready.put((req, ctx, None, e))

    def run(self, requests: Sequence[Request]) -> ServingStats:
        stats = ServingStats()
        pending = deque(sorted(requests, key=lambda r: r.arrival_s))
        ready: "_queue.Queue" = _queue.Queue()
        B = self.make_batch(self.device)
        B.open(self.slots, self.storage, rr_interval=self.rr_interval, graph_iters=self.graph_iters)
        idle: List = []          # pooled contexts not holding a request
        every: List = []         # every context made, closed at the end
        running = {}             # slot -> (request, context, system index)
        building_est = [0]       # estimated bytes of admitted systems still being built
        in_use = [0]             # estimated bytes of every admitted request not yet retired
        building = [0]
        free0 = self.free_memory(self.device)
        t0 = time.perf_counter()

        def fits(req: Request) -> bool:
            if in_use[0] == 0:
                return True      # alone on the device: admit (a system too large fails with its error)
            if in_use[0] + req.est_bytes > self.budget:
                return False
            free = self.free_memory(self.device) + sum(c.device_bytes for c in idle) - self.reserve
            return req.est_bytes <= free - building_est[0]

        def take(item):
            req, ctx, P, err = item
            building[0] -= 1
            building_est[0] -= req.est_bytes
            if ctx is not None and ctx not in every:
                every.append(ctx)
            if err is not None:
                stats.fail(req.rid, repr(err))
                in_use[0] -= req.est_bytes
                if ctx is not None:
                    idle.append(ctx)
                return
            k = None
            try:
                k = B.add_system(ctx)
                slot = B.submit(k, P.b_run, None, self.max_iter, self.tol)
            except Exception as e:
                stats.fail(req.rid, repr(e))
                if k is not None:
                    B.remove_system(k)
                in_use[0] -= req.est_bytes
                idle.append(ctx)
                return
            running[slot] = (req, ctx, k)
            stats.max_in_flight = max(stats.max_in_flight, len(running))

        with ThreadPoolExecutor(max_workers=self.builders) as ex:
            try:
                while pending or building[0] or running:
                    now = time.perf_counter() - t0
                    while pending and pending[0].arrival_s <= now and building[0] < self.builders:
                        req = pending[0]
                        if not fits(req):
                            break
                        pending.popleft()
                        building[0] += 1
                        building_est[0] += req.est_bytes
                        in_use[0] += req.est_bytes
                        ex.submit(self._build, req, idle.pop() if idle else None, ready)
                    while True:
                        try:
                            take(ready.get_nowait())
                        except _queue.Empty:
                            break
                    stats.peak_bytes = max(stats.peak_bytes, free0 - self.free_memory(self.device))
                    if running:
                        stopped, _ = B.step()
                        if stopped:
                            _, res = B.retire(stopped)
                            t = time.perf_counter() - t0
                            for s, r in zip(stopped, res):
                                req, ctx, k = running.pop(s)
                                B.remove_system(k)
                                idle.append(ctx)
                                in_use[0] -= req.est_bytes
                                if r.converged:
                                    stats.latencies_ms.append((t - req.arrival_s) * 1e3)
                                    stats.iters.append(r.iters)
                                    stats.service_ms.append(r.solve_ms)
                                else:
                                    stats.fail(req.rid, f"{r.status} after {r.iters} iterations")
                        continue
                    # nothing on the device: wait for a built system or the next arrival
                    wait = 0.05
                    if pending and building[0] < self.builders:
                        wait = min(wait, max(0.0, pending[0].arrival_s - (time.perf_counter() - t0)))
                    try:
                        take(ready.get(timeout=max(wait, 1e-4)))
                    except _queue.Empty:
                        pass
            finally:
                stats.elapsed_s = time.perf_counter() - t0
        B.close()
        for c in every:
            c.close()
        return stats


def serve_sharded(requests: Sequence[Request], loop: "ServingLoop", dist=None) -> dict:
    """The serving loop on several GPUs, one process per GPU: rank r serves
    every world-th request in arrival order (its share of the stream, at the
    original arrival times) with `loop` on its own device, and the ranks
    exchange their results once at the end (no collective on the data path).
    Returns the summary over all requests on every rank: solves, failures,
    p50 / p99 latency over all of them, solves/s over the slowest rank's
    elapsed time, and each rank's solves and peak device bytes."""
    queue = sorted(requests, key=lambda r: r.arrival_s)
    rank = dist.get_rank() if dist is not None else 0
    world = dist.get_world_size() if dist is not None else 1
    mine = queue[rank::world]
    st = loop.run(mine)
    part = {"latencies_ms": st.latencies_ms, "iters": st.iters, "failed": st.failed, "elapsed_s": st.elapsed_s,
            "peak_bytes": st.peak_bytes}
    parts = [part]
    if dist is not None and world > 1:
        parts = [None] * world
        dist.all_gather_object(parts, part)
    lat = [v for p in parts for v in p["latencies_ms"]]
    iters = [v for p in parts for v in p["iters"]]
    elapsed = max(p["elapsed_s"] for p in parts)
    return {"ranks": world, "solves": len(lat), "failed": sum(p["failed"] for p in parts),
            "elapsed_s": round(elapsed, 3),
            "solves_per_s": round(len(lat) / elapsed, 3) if elapsed > 0 else 0.0,
            "p50_ms": round(percentile(lat, 50), 3), "p99_ms": round(percentile(lat, 99), 3),
            "mean_iters": round(statistics.mean(iters), 1) if iters else 0.0,
            "solves_per_rank": [len(p["latencies_ms"]) for p in parts],
            "peak_device_bytes_per_rank": [p["peak_bytes"] for p in parts]}


def estimate_device_bytes(n: int, nnz: int) -> int:
    """Device memory of one resident system (FP64 + FP32 copies of A in CSR and
    SELL-32, the IC(0) factor in both layouts, about a dozen vectors, and a
    batch slot's nine vectors): a
    conservative linear model used for admission."""
    nnz_l = (nnz + n) // 2
    return int(nnz * 40 + nnz_l * 56 + n * 300 + (8 << 20))
