"""Replica orchestration across ranks (world size 2, gloo on CPU).

The GPU benchmark runs one independent solve per GPU. Its only cross-rank
steps are barriers, a MAX of the elapsed time and a SUM of the completed
solves (iccg_b200.replicas). These run here with two CPU processes. Each
rank solves a small system of its own with the oracle, so the ranks
really do different amounts of work.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import time
    from datetime import timedelta

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import iccg_b200.problems as pb
        from iccg_b200.replicas import timed_replicas, max_over_ranks
        from oracle import bindings as ob

        # rank r: a 2D Poisson system of side 24 + 8 r, solved by the oracle
        P = pb.config_small_mc(24 + 8 * rank, seed=rank)
        A = P.A_run
        ic0 = ob.OracleIC0(A.n, A.rowptr, A.colind, A.val, 0.0)
        steps = 2 + rank
        iters = []

        def run():
            t0 = time.perf_counter()
            for _ in range(steps):
                x, it, rel, cv, _ = ob.cg(A.n, A.rowptr, A.colind, A.val, P.b_run, np.zeros(A.n), 2, 1000, 1e-8,
                                          ic0, P.sched)
                assert cv
                iters.append(it)
            time.sleep(0.05 * (rank + 1))  # make the slower rank unambiguous
            return (time.perf_counter() - t0) * 1e3

        tr = timed_replicas(run, steps, dist=dist, device="cpu")
        out[rank] = (tr.ms, tr.units, tr.world, max_over_ranks(float(rank), dist=dist, device="cpu"), iters[0])
    finally:
        dist.destroy_process_group()


def test_replicas_two_ranks_gloo():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = dict(out)
    assert set(res) == {0, 1}
    ms0, units0, w0, mx0, it0 = res[0]
    ms1, units1, w1, mx1, it1 = res[1]
    # every rank reports the same reduced figures
    assert ms0 == ms1 and units0 == units1 and w0 == w1 == world
    # units summed over ranks (2 + 3 solves), time = the slowest rank's
    assert units0 == 5
    assert ms0 >= 100.0  # rank 1 slept 0.1 s inside its timed region
    assert mx0 == mx1 == 1.0
    assert it0 > 0 and it1 > 0


def test_replicas_single_process():
    from iccg_b200.replicas import timed_replicas, max_over_ranks
    tr = timed_replicas(lambda: 12.5, 3)
    assert (tr.ms, tr.units, tr.world) == (12.5, 3, 1)
    assert abs(tr.units_per_s - 240.0) < 1e-9
    assert max_over_ranks(4.0) == 4.0


# ---------------------------------------------------------------------------
# serving on several GPUs: requests sharded over ranks
# ---------------------------------------------------------------------------
class _FakeCtx:
    def __init__(self, device):
        self.device = device

    def close(self):
        pass


class _FakeSystem:
    """Stands in for a resident system: a short sleep as its solve."""

    def __init__(self, P, device, storage, ctx=None):
        self.P = P

    @property
    def device_bytes(self):
        return 1000 * self.P.n

    def solve(self, b, tol):
        import time
        from types import SimpleNamespace
        time.sleep(0.002)
        return np.zeros_like(b), SimpleNamespace(converged=True, iters=7), 2.0

    def close(self):
        pass


def _requests(count):
    from types import SimpleNamespace
    import iccg_b200.batch as bt
    return [bt.Request(i, 0.005 * i, (lambda i=i: SimpleNamespace(n=10 + i, b_run=np.zeros(10 + i))), 1 << 20)
            for i in range(count)]


def _serve_rank(rank, world, port, out):
    from datetime import timedelta

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import iccg_b200.batch as bt
        loop = bt.ThreadedServingLoop(budget_bytes=1 << 30, workers=2, make_system=_FakeSystem, make_context=_FakeCtx)
        out[rank] = bt.serve_sharded(_requests(11), loop, dist=dist)
    finally:
        dist.destroy_process_group()


def test_serving_sharded_over_two_ranks_gloo():
    """Each rank serves every other request of the stream at its arrival
    time; both ranks end with the summary over all 11 requests."""
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_serve_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    s0, s1 = out[0], out[1]
    assert s0 == s1
    assert s0["ranks"] == 2 and s0["solves"] == 11 and s0["failed"] == 0
    assert s0["solves_per_rank"] == [6, 5]
    assert s0["p99_ms"] >= s0["p50_ms"] > 0 and s0["solves_per_s"] > 0
    assert s0["mean_iters"] == 7.0
    assert all(b > 0 for b in s0["peak_device_bytes_per_rank"])


def test_serving_sharded_single_process():
    import iccg_b200.batch as bt
    loop = bt.ThreadedServingLoop(budget_bytes=1 << 30, workers=3, make_system=_FakeSystem, make_context=_FakeCtx)
    s = bt.serve_sharded(_requests(7), loop)
    assert s["ranks"] == 1 and s["solves"] == 7 and s["solves_per_rank"] == [7] and s["failed"] == 0
