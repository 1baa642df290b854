"""The persistent IC(0) apply (one launch per apply, work items taken from a
ticket counter, per-item dependency flags) against the per-level kernels
and the oracle.

FP64: the same bits as the per-level kernels (which are bit-exact with the
reference) for applies, SpMV-free fused and plain solves, on every ordering
kind: multicolor, ABMC with linear and breadth-first blocks (in-unit
entries on any earlier step), units of 32 and 64 rows, the natural order's
level sets, k-NN graphs and ragged tiny systems.  FP32 storage: applies to
FP32 rounding of the per-level result and solves to the true residual.
Many launches in a row (the ticket counter and done flags carry over from
launch to launch) must keep giving the same bits.
"""
import numpy as np
import pytest

import iccg_b200 as ib
import iccg_b200.problems as pb
from oracle import bindings as ob
from _util import rel_err

pytestmark = pytest.mark.gpu

SYSTEMS = {
    "mc2d": lambda: pb.config_small_mc(100, seed=1),
    "abmc_lin": lambda: pb.config_abmc_aniso(40, 16, "linear"),
    "abmc_bfs": lambda: pb.config_abmc_aniso(40, 16, "bfs"),
    "abmc_b32_lin": lambda: pb.config_abmc_aniso(40, 32, "linear"),
    "d27_mc": lambda: pb.config_diffusion27(24, "piccg"),
    "d27_abmc8": lambda: pb.config_diffusion27(24, "abmc", 8),
    "d27_abmc32": lambda: pb.config_diffusion27(24, "abmc", 32),
    "d27_abmc64": lambda: pb.config_diffusion27(20, "abmc", 64),
    "p2d_abmc64": lambda: pb.make(pb.poisson2d(96), "abmc", block_size=64, blocking="bfs", seed=4),
    "natural": lambda: pb.make(pb.laplace3d_aniso(12), "iccg", seed=1),
    "knn": lambda: pb.config_knn(8000, seed=5, block_size=16),
    "tiny": lambda: pb.make(pb.laplace3d_aniso(3), "abmc", block_size=16, seed=4),
}


# systems whose every level fits the stage budget (FP32 storage; FP64's
# backward batches park their gathered values too, and may not fit)
PERSISTENT = {"mc2d", "abmc_lin", "abmc_bfs", "abmc_b32_lin", "d27_mc", "d27_abmc8", "natural", "knn", "tiny"}


def _ctx(P):
    ctx = ib.Context(0)
    ctx.upload(P.A_run)
    ctx.set_schedule(P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    ctx.set_option(ib.OPT_PERSIST, 1)
    return ctx


@pytest.mark.parametrize("which", sorted(SYSTEMS))
def test_gpu_persistent_apply_equals_per_level_kernels(which):
    P = SYSTEMS[which]()
    ctx = _ctx(P)
    # the persistent apply takes the staged batches: systems where a level's
    # group exceeds the stage budget keep the per-level kernels
    for st in (ib.STORE_FP64, ib.STORE_FP32):
        plan = {k for k, _ in ctx.sweep_plan(st, True)}
        assert plan == {"persistent"} or "persistent" not in plan
        if which in PERSISTENT and st == ib.STORE_FP32:
            assert plan == {"persistent"}, plan
    r = ib.gen_uniform(P.A_run.n, 31)
    out = {}
    for persist in (1, 0):
        ctx.set_option(ib.OPT_PERSIST, persist)
        res = {}
        for st in (ib.STORE_FP64, ib.STORE_FP32):
            z = ctx.apply(r, st)
            sol = {}
            for mode in ((ib.MODE_FUSED, ib.MODE_PLAIN) if st == ib.STORE_FP64 else (ib.MODE_FUSED,)):
                x = np.zeros(P.A_run.n)
                rr = ctx.solve(P.b_run, x, 10000, 1e-8, storage=st, mode=mode)
                sol[mode] = (x, rr)
            res[st] = (z, sol)
        out[persist] = res
    a, b = out[1][ib.STORE_FP64], out[0][ib.STORE_FP64]
    assert np.array_equal(a[0], b[0])
    ic0 = ob.OracleIC0(P.A_run.n, P.A_run.rowptr, P.A_run.colind, P.A_run.val, 0.0)
    assert np.array_equal(a[0], ic0.apply(r, P.sched))
    for mode in (ib.MODE_FUSED, ib.MODE_PLAIN):
        (xa, ra), (xb, rb) = a[1][mode], b[1][mode]
        assert ra.converged and ra.iters == rb.iters
        assert np.array_equal(xa, xb)
    a, b = out[1][ib.STORE_FP32], out[0][ib.STORE_FP32]
    assert rel_err(a[0], b[0]) < 1e-5
    (xa, ra), (xb, rb) = a[1][ib.MODE_FUSED], b[1][ib.MODE_FUSED]
    assert ra.converged and ra.true_rel_resid <= 1e-8 and abs(ra.iters - rb.iters) <= 2
    assert rel_err(xa, xb) < 1e-6
    ctx.close()


@pytest.mark.parametrize("which", ["abmc_bfs", "d27_mc"])
def test_gpu_persistent_launches_in_a_row_keep_their_bits(which):
    """Forty applies and solves in a row, alternating FP64 and FP32 storage
    (separate ticket counters) and dropping the graphs in between: the
    counters and flags left by each launch must never let a later launch
    read an item before it is done."""
    P = SYSTEMS[which]()
    ctx = _ctx(P)
    r = ib.gen_uniform(P.A_run.n, 5)
    z64 = ctx.apply(r, ib.STORE_FP64)
    z32 = ctx.apply(r, ib.STORE_FP32)
    x0 = np.zeros(P.A_run.n)
    r0 = ctx.solve(P.b_run, x0, 10000, 1e-8, storage=ib.STORE_FP64)
    for k in range(40):
        assert np.array_equal(ctx.apply(r, ib.STORE_FP64), z64)
        assert np.array_equal(ctx.apply(r, ib.STORE_FP32), z32)
        if k % 8 == 0:
            ctx.set_option(ib.OPT_PDL, (k // 8) % 2)   # drops the captured graphs too
            x = np.zeros(P.A_run.n)
            rr = ctx.solve(P.b_run, x, 10000, 1e-8, storage=ib.STORE_FP64)
            assert rr.iters == r0.iters and np.array_equal(x, x0)
    ctx.close()


def test_gpu_persistent_solve_stops_like_the_reference():
    """max_iter caps and an iteration-0 convergence with the update fused into
    the persistent launch: the deferred stop lands on the same iteration as
    the reference's."""
    P = pb.config_small_mc(16)
    ctx = _ctx(P)
    ic0 = ob.OracleIC0(P.A_run.n, P.A_run.rowptr, P.A_run.colind, P.A_run.val, 0.0)
    for cap in (1, 2, 5, 9):
        xo, ito, relo, cvo, _ = ob.cg(P.A_run.n, P.A_run.rowptr, P.A_run.colind, P.A_run.val, P.b_run,
                                      np.zeros(P.A_run.n), 2, cap, 1e-8, ic0, P.sched)
        x = np.zeros(P.A_run.n)
        res = ctx.solve(P.b_run, x, cap, 1e-8)
        assert res.iters == ito and not res.converged and res.status == "max_iter"
        assert rel_err(x, xo) <= 1e-10
    # converged before the first iteration: b = 0
    x = np.zeros(P.A_run.n)
    res = ctx.solve(np.zeros(P.A_run.n), x, 100, 1e-8)
    assert res.converged and res.iters == 0 and not x.any()
    # the mixed form's true-residual check at the end, through the fused launch
    for gi in (1, 3, 8):
        x = np.zeros(P.A_run.n)
        res = ctx.solve(P.b_run, x, 10000, 1e-8, storage=ib.STORE_FP32, graph_iters=gi)
        assert res.converged and res.true_rel_resid <= 1e-8
    ctx.close()
