"""Replicas on several GPUs (one process per GPU, torch.distributed).

A single preconditioned CG solve does not shard without a halo exchange and
two all-reduces per iteration.  So several GPUs run independent replicas:
each rank solves its own system, and there is no collective on the data path.
The only cross-rank steps are these:

* a barrier on each side of the timed region;
* a MAX reduction of the per-rank elapsed time, since the job ends with its
  slowest rank;
* a SUM reduction of the units (solves) the ranks completed.

Whole-job throughput is the summed units divided by that maximum time.  The
same code runs over NCCL on GPUs and over gloo on CPU (the tests).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, Optional


@dataclass
class ReplicaTiming:
    ms: float          # slowest rank's elapsed ms for the timed region
    units: float       # units completed by all ranks together
    world: int

    @property
    def units_per_s(self) -> float:
        return self.units / (self.ms * 1e-3) if self.ms > 0 else 0.0


def _reduce(dist, value: float, op, device) -> float:
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def timed_replicas(run: Callable[[], float], units: float, dist=None, device=None,
                   sync: Optional[Callable[[], None]] = None) -> ReplicaTiming:
    """Times `run` on every rank between barriers.

    `run()` does the timed work and returns its elapsed ms (CUDA events on
    the GPU). `units` is what this rank completed. `sync` (e.g.
    torch.cuda.synchronize) runs after each barrier. `dist` is
    torch.distributed or None for a single process; `device` holds the
    reduction tensors ("cuda" for NCCL, "cpu" for gloo).
    """
    if dist is not None:
        dist.barrier()
    if sync:
        sync()
    ms = run()
    if sync:
        sync()
    if dist is None:
        return ReplicaTiming(ms=ms, units=units, world=1)
    dist.barrier()
    world = dist.get_world_size()
    ms_max = _reduce(dist, ms, dist.ReduceOp.MAX, device)
    units_all = _reduce(dist, units, dist.ReduceOp.SUM, device)
    return ReplicaTiming(ms=ms_max, units=units_all, world=world)


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The largest `value` over all ranks (the value itself for one process)."""
    if dist is None:
        return value
    return _reduce(dist, value, dist.ReduceOp.MAX, device)
