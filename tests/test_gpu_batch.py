"""The earlier many-streams batch form and both serving loops
(iccg_b200.batch) on the GPU.

Several systems solve at once, one context and stream each. The solver's
arithmetic does not depend on what runs beside it, so every result must be
bit-identical to the same solve run alone.  The serving loops serve every
request of a small kNN stream under a device-memory budget.
"""
import numpy as np
import pytest

import iccg_b200 as ib
import iccg_b200.batch as bt
import iccg_b200.problems as pb

pytestmark = pytest.mark.gpu


def _systems():
    out = []
    for i, side in enumerate((20, 33, 48, 27)):
        out.append(pb.make(pb.poisson2d(side), "piccg", seed=i))
    for i, side in enumerate((10, 13, 16)):
        out.append(pb.make(pb.laplace3d_aniso(side, 1.0), "piccg", seed=10 + i))
    out.append(pb.config_abmc_aniso(14, 16, "bfs", seed=3))
    return out


@pytest.mark.parametrize("storage", [ib.STORE_FP64, ib.STORE_FP32])
def test_batch_results_equal_alone(storage):
    probs = _systems()
    rhs = [[pb.with_rhs(P, seed=100 * k + 7).b_run.copy() for k in range(2)] for P in probs]
    systems = [bt.ResidentSystem(P, storage=storage) for P in probs]
    try:
        alone = bt.solve_batch(systems, rhs, threads=1, keep_x=True)
        mixed = bt.solve_batch(systems, rhs, threads=6, keep_x=True)
        assert len(alone) == len(mixed) == 2 * len(probs)
        key = lambda r: (r.system, r.rhs)
        for a, m in zip(sorted(alone, key=key), sorted(mixed, key=key)):
            assert a.converged and m.converged
            assert a.iters == m.iters
            assert np.array_equal(a.x, m.x), (a.system, a.rhs)
            assert m.true_rel_resid <= 1e-8
    finally:
        for s in systems:
            s.close()


def test_serving_loop_admits_under_budget():
    sizes = [1000, 2500, 4000, 1500, 3000, 2000, 5000, 1200]
    reqs = []
    for i, npts in enumerate(sizes):
        est = bt.estimate_device_bytes(npts, 18 * npts)
        reqs.append(bt.Request(i, 0.02 * i, (lambda npts=npts, i=i: pb.config_knn(npts, seed=i)), est))
    budget = 3 * max(r.est_bytes for r in reqs)
    for loop in (bt.ServingLoop(budget_bytes=budget, builders=4, slots=8, graph_iters=2),
                 bt.ThreadedServingLoop(budget_bytes=budget, workers=4)):
        st = loop.run(reqs)
        s = st.summary()
        assert s["solves"] == len(sizes) and s["failed"] == 0, s
        assert s["p99_ms"] >= s["p50_ms"] > 0
        assert s["solves_per_s"] > 0


@pytest.mark.parametrize("storage", [ib.STORE_FP64, ib.STORE_FP32])
def test_reused_context_gives_the_same_bits_as_a_fresh_one(storage):
    """A serving worker loads system after system into one context, whose
    device buffers only grow.  A smaller system loaded after a larger one,
    and the larger one loaded again, solve to the same bits as in fresh
    contexts."""
    big = pb.config_abmc_aniso(32, 16, "bfs", seed=1)
    small = pb.make(pb.poisson2d(40), "piccg", seed=2)
    fresh = {}
    for name, P in (("big", big), ("small", small)):
        s = bt.ResidentSystem(P, storage=storage)
        fresh[name] = s.solve(P.b_run)[0]
        s.close()
    ctx = ib.Context(0)
    try:
        for name, P in (("big", big), ("small", small), ("big", big)):
            s = bt.ResidentSystem(P, storage=storage, ctx=ctx)
            x, res, _ = s.solve(P.b_run)
            s.close()
            assert res.converged
            assert np.array_equal(x, fresh[name]), name
    finally:
        ctx.close()
