"""Per-matrix tuning: the ordering of a system and the kernel options of a
context, chosen by timing solves on the device.

The reference takes its coloring or ABMC blocking from external files
(run_mc.sh, run_abmc.sh) and runs one OpenMP code path. On the GPU the best
ordering depends on the matrix: more, smaller units give more parallel
chains per color but more colors and iterations. So the tuner times the
candidates on the matrix itself.

* ``tune_ordering(A, ...)`` builds every candidate ordering (multicolor,
  ABMC with each block size and blocking) with this package's generators. It times one
  full solve of each on the device, after a warm-up solve, and returns the
  fastest ``Problem`` with the table of timings. Candidates differ in
  iteration count as well as in speed per iteration; the tuner compares
  time to tolerance.
* ``tune_batch(matrices, ...)`` picks the ordering of every system of a
  batch: the systems are grouped into classes (by default the rounded
  entries per row and the power of two of the row count), the ordering of
  the largest system of each class is tuned as above, and every system of
  the class is built with it.
* ``tune_kernels(ctx, b_run, ...)`` chooses the context options of a built
  system by coordinate search: for each option in turn it keeps the value
  with the lowest median solve time, the others held at their best so far.
  The options are the sweep kernel (staged or per-slice), the staged
  kernel's buffers per CTA and shared-memory budget, and programmatic
  dependent launch. With
  FP64 storage every choice gives the same bits. With FP32 storage the
  staged and per-slice sweeps round differently (reciprocal pivots against
  divisions), so the tuned result can differ in the last bits from an
  untuned one. Both meet the tolerance.

Timing goes through a ``timer`` callable that returns (ms, iterations,
converged) for a candidate (by default the median device time of solves on
the GPU), so the selection logic can be driven without a GPU.
"""
from __future__ import annotations

import statistics
from dataclasses import dataclass, field
from typing import Callable, Dict, Hashable, List, Optional, Sequence, Tuple

import numpy as np

from . import (CRS, MODE_FUSED, OPT_DEFER_X, OPT_EARLY, OPT_FUSE_UPDATE, OPT_PDL, OPT_UPDATE_CHAIN, OPT_PERSIST, OPT_SPMV_PACK, OPT_STAGE_BUFS,
               OPT_SPMV_TPR, OPT_STAGE_KB, OPT_STAGE_ROWS, OPT_SWEEP, PRECOND_IC0,
               STORE_FP32, Context)
from .problems import Problem, make

# (variant, block size, blocking) candidates: multicolor, and ABMC with 8, 16,
# 32 rows per block grown by breadth-first search, or 16 and 32 consecutive
# rows (linear blocking: on structured grids it can need far fewer colors)
ORDERINGS: Tuple[Tuple[str, int, str], ...] = (("piccg", 0, "bfs"), ("abmc", 8, "bfs"), ("abmc", 16, "bfs"),
                                               ("abmc", 32, "bfs"), ("abmc", 16, "linear"),
                                               ("abmc", 32, "linear"))

# the candidates per class of a batch: small systems, so the 8-row blocks
# (more parallel chains) are in and the linear blockings are not
BATCH_ORDERINGS: Tuple[Tuple[str, int, str], ...] = (("piccg", 0, "bfs"), ("abmc", 8, "bfs"), ("abmc", 16, "bfs"),
                                                     ("abmc", 32, "bfs"))

# option -> candidate values, in the order they are tried (the first is the default)
KERNEL_OPTIONS: Tuple[Tuple[int, Tuple[int, ...]], ...] = (
    (OPT_PERSIST, (0, 1)),
    (OPT_SWEEP, (0, 1)),
    (OPT_STAGE_BUFS, (1, 2)),
    (OPT_STAGE_KB, (0, 160, 112, 80)),
    (OPT_STAGE_ROWS, (256, 512, 128)),
    (OPT_PDL, (1, 0)),
    (OPT_EARLY, (1, 0, 3)),
    (OPT_SPMV_PACK, (1, 0)),
    (OPT_SPMV_TPR, (1, 2, 4)),
    (OPT_FUSE_UPDATE, (0, 1)),
    (OPT_DEFER_X, (0, 1)),
    (OPT_UPDATE_CHAIN, (0, 1)),
)
OPTION_NAMES = {OPT_PERSIST: "persist", OPT_SWEEP: "sweep", OPT_STAGE_BUFS: "stage_bufs", OPT_STAGE_KB: "stage_kb",
                OPT_PDL: "pdl", OPT_SPMV_PACK: "spmv_pack", OPT_FUSE_UPDATE: "fuse_update", OPT_DEFER_X: "defer_x",
                OPT_STAGE_ROWS: "stage_rows", OPT_SPMV_TPR: "spmv_tpr", OPT_EARLY: "early",
                OPT_UPDATE_CHAIN: "update_chain"}


@dataclass
class Trial:
    label: str
    ms: float
    iters: int
    converged: bool


@dataclass
class TuneResult:
    best: str
    trials: List[Trial] = field(default_factory=list)
    choice: Dict = field(default_factory=dict)

    def table(self) -> List[dict]:
        return [{"candidate": t.label, "ms": round(t.ms, 4), "iters": t.iters, "converged": t.converged}
                for t in self.trials]


def _label(variant: str, block: int, blocking: str = "bfs") -> str:
    if variant == "piccg":
        return "mc"
    return f"abmc{block}" + ("" if blocking == "bfs" else f"_{blocking}")


def _solve_time(ctx: Context, b_run: np.ndarray, storage: int, tol: float, reps: int) -> Tuple[float, int, bool]:
    """Median device ms of `reps` solves after one warm-up; iterations and
    convergence of the last."""
    ms, res = [], None
    for i in range(reps + 1):
        x = np.zeros(b_run.shape[0])
        res = ctx.solve(b_run, x, 10000, tol, mode=MODE_FUSED, storage=storage)
        if i:
            ms.append(res.solve_ms)
    return statistics.median(ms), res.iters, bool(res.converged)


def pick(trials: Sequence[Trial]) -> Trial:
    """The fastest converged trial (ties: the first); if none converged, the
    fastest."""
    ok = [t for t in trials if t.converged]
    pool = ok if ok else list(trials)
    return min(pool, key=lambda t: t.ms)


def tune_ordering(A: CRS, candidates: Sequence[Tuple] = ORDERINGS, storage: int = STORE_FP32,
                  tol: float = 1e-8, seed: int = 0, device: int = 0, reps: int = 1,
                  timer: Optional[Callable[[Problem], Tuple[float, int, bool]]] = None) -> Tuple[Problem, TuneResult]:
    """Builds each candidate ordering of A (the original, unpermuted matrix)
    and returns the one whose solve to `tol` is fastest, with the timings.
    A candidate is (variant, block size[, blocking]), blocking "bfs" when
    omitted. `timer(P)` returns (ms, iterations, converged) for a built
    problem; the default uploads P to a fresh context on `device` and times
    `reps` solves."""

    def device_timer(P: Problem) -> Tuple[float, int, bool]:
        ctx = Context(device)
        try:
            ctx.upload(P.A_run)
            ctx.set_schedule(P.sched)
            ctx.build(PRECOND_IC0, 0.0, auto_shift=True)
            return _solve_time(ctx, P.b_run, storage, tol, reps)
        finally:
            ctx.close()

    timer = timer or device_timer
    trials: List[Trial] = []
    built: Dict[str, Problem] = {}
    for cand in candidates:
        variant, block = cand[0], cand[1]
        blocking = cand[2] if len(cand) > 2 else "bfs"
        label = _label(variant, block, blocking)
        P = make(A, variant, block_size=max(block, 1), blocking=blocking, seed=seed, name=label)
        ms, iters, conv = timer(P)
        trials.append(Trial(label, ms, iters, conv))
        built[label] = P
    best = pick(trials)
    res = TuneResult(best=best.label, trials=trials,
                     choice={"ordering": best.label, "ms": best.ms, "iters": best.iters})
    return built[best.label], res


def tune_kernels(ctx: Context, b_run: np.ndarray, storage: int = STORE_FP32, tol: float = 1e-8, reps: int = 2,
                 options: Sequence[Tuple[int, Sequence[int]]] = KERNEL_OPTIONS,
                 timer: Optional[Callable[[], Tuple[float, int, bool]]] = None) -> TuneResult:
    """Coordinate search over the context options of a built system; leaves
    the best values set on `ctx` and returns the timings.  `timer()` times
    the current settings (default: `reps` solves of b_run after a warm-up)."""
    timer = timer or (lambda: _solve_time(ctx, b_run, storage, tol, reps))
    current = {opt: vals[0] for opt, vals in options}
    for opt, v in current.items():
        ctx.set_option(opt, v)
    trials: List[Trial] = []
    best_ms = None
    for opt, vals in options:
        scored = []
        for v in vals:
            ctx.set_option(opt, v)
            ms, iters, conv = timer()
            label = ",".join(f"{OPTION_NAMES.get(o, o)}={current[o] if o != opt else v}" for o, _ in options)
            t = Trial(label, ms, iters, conv)
            trials.append(t)
            scored.append((t, v))
        win = pick([t for t, _ in scored])
        current[opt] = next(v for t, v in scored if t is win)
        ctx.set_option(opt, current[opt])
        best_ms = win.ms
    choice = {OPTION_NAMES.get(o, str(o)): v for o, v in current.items()}
    choice["ms"] = best_ms
    return TuneResult(best=",".join(f"{k}={v}" for k, v in choice.items() if k != "ms"), trials=trials,
                      choice=choice)


def batch_class(A: CRS) -> Tuple[int, int]:
    """Default class of a batch system: (rounded entries per row, bit length
    of the row count), e.g. every 2D 5-point system of 2 049 to 4 096 rows."""
    n = max(A.n, 1)
    return int(round(A.nnz / n)), int(n - 1).bit_length()


def tune_batch(matrices: Sequence[CRS], classes: Optional[Sequence[Hashable]] = None,
               candidates: Sequence[Tuple] = BATCH_ORDERINGS, storage: int = STORE_FP32, tol: float = 1e-8,
               seeds: Optional[Sequence[int]] = None, device: int = 0, reps: int = 1,
               timer: Optional[Callable[[Problem], Tuple[float, int, bool]]] = None
               ) -> Tuple[List[Problem], List[dict]]:
    """Orderings for the systems of a batch (original, unpermuted matrices).
    Systems with the same class (`classes[i]`, default `batch_class`) share
    one choice: the one `tune_ordering` makes for the class's largest system.
    Returns the built problems, in the order of `matrices`, and one row per
    class: its key, members, the system tuned and the timings."""
    m = len(matrices)
    keys = list(classes) if classes is not None else [batch_class(A) for A in matrices]
    if len(keys) != m:
        raise ValueError("one class per matrix")
    seeds = list(seeds) if seeds is not None else list(range(m))
    if len(seeds) != m:
        raise ValueError("one seed per matrix")
    members: Dict[Hashable, List[int]] = {}
    for i, k in enumerate(keys):
        members.setdefault(k, []).append(i)
    out: List[Optional[Problem]] = [None] * m
    rows = []
    for key, idx in members.items():
        rep = max(idx, key=lambda i: (matrices[i].n, -i))
        P, res = tune_ordering(matrices[rep], candidates, storage=storage, tol=tol, seed=seeds[rep], device=device,
                               reps=reps, timer=timer)
        best = next(c for c in candidates if _label(c[0], c[1], c[2] if len(c) > 2 else "bfs") == res.best)
        blocking = best[2] if len(best) > 2 else "bfs"
        for i in idx:
            out[i] = P if i == rep else make(matrices[i], best[0], block_size=max(best[1], 1), blocking=blocking,
                                             seed=seeds[i], name=res.best)
        rows.append({"class": key, "systems": len(idx), "tuned_on_rows": matrices[rep].n, "choice": res.best,
                     "trials": res.table()})
    return [P for P in out if P is not None], rows
