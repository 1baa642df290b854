"""Per-matrix tuning on the GPU: the ordering tuner returns a converged
candidate built like any other problem, and the kernel-option tuner leaves
options that keep an FP64 solve's bits (every kernel choice does)."""
import numpy as np
import pytest

import iccg_b200 as ib
import iccg_b200.autotune as at
import iccg_b200.problems as pb

pytestmark = pytest.mark.gpu


def test_gpu_tune_ordering_returns_a_converged_candidate():
    A = pb.gen_diffusion27(20, 20, 20, 1e4, 3)
    P, res = at.tune_ordering(A, storage=ib.STORE_FP32, reps=1)
    assert len(res.trials) == len(at.ORDERINGS)
    assert all(t.converged for t in res.trials), res.table()
    best = min(res.trials, key=lambda t: t.ms)
    assert res.best == best.label == P.name
    ctx = ib.Context(0)
    ctx.upload(P.A_run)
    ctx.set_schedule(P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    x = np.zeros(P.A_run.n)
    r = ctx.solve(P.b_run, x, 10000, 1e-8, storage=ib.STORE_FP32)
    assert r.converged and r.true_rel_resid <= 1e-8
    ctx.close()


def test_gpu_tune_kernels_keeps_fp64_bits():
    P = pb.config_diffusion27(24, "piccg")
    ctx = ib.Context(0)
    ctx.upload(P.A_run)
    ctx.set_schedule(P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    x0 = np.zeros(P.A_run.n)
    r0 = ctx.solve(P.b_run, x0, 10000, 1e-8, storage=ib.STORE_FP64)
    res = at.tune_kernels(ctx, P.b_run, storage=ib.STORE_FP32, reps=1)
    assert res.choice["sweep"] in (0, 1) and res.choice["stage_kb"] in (0, 160, 112, 80)
    assert res.choice["pdl"] in (0, 1) and res.choice["stage_bufs"] in (1, 2) and res.choice["persist"] in (0, 1)
    assert len(res.trials) == sum(len(v) for _, v in at.KERNEL_OPTIONS)
    x1 = np.zeros(P.A_run.n)
    r1 = ctx.solve(P.b_run, x1, 10000, 1e-8, storage=ib.STORE_FP64)
    assert r1.iters == r0.iters and np.array_equal(x1, x0)
    x2 = np.zeros(P.A_run.n)
    r2 = ctx.solve(P.b_run, x2, 10000, 1e-8, storage=ib.STORE_FP32)
    assert r2.converged and r2.true_rel_resid <= 1e-8
    ctx.close()
