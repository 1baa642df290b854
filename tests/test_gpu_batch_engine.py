"""The batched solve engine (iccg_batch, ib.Batch) on the GPU.

Every CG step of all the batch's solves is one launch over a work list; the
per-row arithmetic and the per-solve reductions are those of a solve alone,
so each solve must give the same bits of x, the same iteration count,
status and residuals as Context.solve on its system alone -- for uneven
systems (2D and 3D, different sizes, level counts and orderings), several
right-hand sides per system, FP64 and the mixed form, solves that stop at
different iterations, a zero right-hand side and iteration caps.
"""
import numpy as np
import pytest

import iccg_b200 as ib
import iccg_b200.problems as pb

pytestmark = pytest.mark.gpu


def _uneven_systems():
    out = []
    for i, side in enumerate((8, 13, 21, 30, 37, 44, 52, 60)):
        out.append(pb.make(pb.poisson2d(side), "piccg", seed=i))
    for i, side in enumerate((4, 6, 9, 11, 14, 17, 20)):
        out.append(pb.make(pb.laplace3d_aniso(side, 1.0), "piccg", seed=20 + i))
    for i, side in enumerate((5, 10, 15, 19)):
        out.append(pb.config_abmc_aniso(side, 16, "linear", seed=40 + i))
    for i, side in enumerate((7, 12, 18)):
        out.append(pb.config_abmc_aniso(side, 16, "bfs", seed=50 + i))
    out.append(pb.config_diffusion27(10, "piccg", seed=60))
    out.append(pb.config_diffusion27(12, "abmc", 8, seed=61))
    return out


def _ctx(P):
    ctx = ib.Context(0)
    ctx.upload(P.A_run)
    ctx.set_schedule(P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    return ctx


def _alone(ctx, b, storage, max_iter=10000, tol=1e-8, rr_interval=50):
    x = np.zeros(ctx.n)
    r = ctx.solve(b, x, max_iter, tol, storage=storage, rr_interval=rr_interval)
    return x, r


def _same(a, b):
    (xa, ra), (xb, rb) = a, b
    assert ra.status == rb.status, (ra, rb)
    assert ra.iters == rb.iters, (ra, rb)
    assert ra.converged == rb.converged
    assert ra.n_replacements == rb.n_replacements
    assert ra.rel_resid == rb.rel_resid
    assert np.array_equal(xa, xb)
    if np.isfinite(rb.true_rel_resid):
        assert ra.true_rel_resid == pytest.approx(rb.true_rel_resid, rel=1e-12, abs=1e-300)


@pytest.mark.parametrize("storage", [ib.STORE_FP64, ib.STORE_FP32])
def test_gpu_batch_equals_solves_alone(storage):
    probs = _uneven_systems()
    assert len(probs) >= 20
    ctxs = [_ctx(P) for P in probs]
    B = ib.Batch(0)
    idx = [B.add_system(c) for c in ctxs]
    systems, bs, xs = [], [], []
    for k, P in enumerate(probs):
        for j in range(2):
            systems.append(idx[k])
            bs.append(pb.with_rhs(P, seed=100 * k + j).b_run.copy())
            xs.append(np.zeros(P.A_run.n))
    # solves of one system side by side, then a shuffled order: same bits
    res = B.solve(systems, bs, xs, 10000, 1e-8, storage=storage)
    for s, (k, b) in enumerate(zip(systems, bs)):
        alone = _alone(ctxs[k], b, storage)
        _same((xs[s], res[s]), alone)
        assert res[s].converged
        assert 0.0 < res[s].solve_ms <= B.device_ms + 1e-6
    perm = np.random.default_rng(1).permutation(len(systems))
    xs2 = [np.zeros_like(xs[s]) for s in perm]
    res2 = B.solve([systems[s] for s in perm], [bs[s] for s in perm], xs2, 10000, 1e-8, storage=storage)
    for t, s in enumerate(perm):
        _same((xs2[t], res2[t]), (xs[s], res[s]))
    # fewer launches than the solves run alone: one per step for all
    assert B.launches > 0
    B.close()
    for c in ctxs:
        c.close()


def test_gpu_batch_mixed_orderings_and_stops():
    probs = [
        pb.config_abmc_aniso(16, 16, "linear", seed=1),
        pb.config_abmc_aniso(16, 16, "bfs", seed=2),
        pb.config_knn(3000, seed=5, block_size=16),
        pb.config_small_mc(24, seed=3),
        pb.config_diffusion27(14, "abmc", 8, seed=4),
    ]
    ctxs = [_ctx(P) for P in probs]
    B = ib.Batch(0)
    for c in ctxs:
        B.add_system(c)
    systems = [0, 1, 2, 3, 4, 3, 0]
    bs = [probs[k].b_run.copy() for k in systems]
    bs[5] = np.zeros(probs[3].A_run.n)             # converged before the first iteration
    x0 = [ib.gen_uniform(len(b), 7 + s) for s, b in enumerate(bs)]
    x0[5] = np.zeros(len(bs[5]))
    for storage in (ib.STORE_FP64, ib.STORE_FP32):
        for max_iter in (10000, 3):
            for tol in (1e-8, 1e-3):
                xs = [x.copy() for x in x0]
                res = B.solve(systems, bs, xs, max_iter, tol, storage=storage, rr_interval=20, graph_iters=4)
                for s, k in enumerate(systems):
                    x = x0[s].copy()
                    r = ctxs[k].solve(bs[s], x, max_iter, tol, storage=storage, rr_interval=20, graph_iters=4)
                    _same((xs[s], res[s]), (x, r))
                    if max_iter == 3 and s != 5:
                        assert res[s].iters == 3 and res[s].status == "max_iter"
                assert res[5].converged and res[5].iters == 0 and not xs[5].any()
    # a batch of one solve with a cap
    x = np.zeros(probs[0].A_run.n)
    r = B.solve([0], [bs[0]], [x], 3, 1e-8)[0]
    assert r.iters == 3 and r.status == "max_iter"
    B.close()
    for c in ctxs:
        c.close()


def test_gpu_batch_rejects_bad_arguments():
    P = pb.config_small_mc(12)
    ctx = _ctx(P)
    B = ib.Batch(0)
    with pytest.raises(ValueError):
        B.solve([0], [P.b_run], [np.zeros(P.A_run.n)])     # no system yet
    k = B.add_system(ctx)
    with pytest.raises(ValueError):
        B.solve([k + 1], [P.b_run], [np.zeros(P.A_run.n)])
    with pytest.raises(ValueError):
        B.solve([k], [P.b_run[:-1]], [np.zeros(P.A_run.n)])
    plain = ib.Context(0)
    plain.upload(P.A_run)
    with pytest.raises(ib.IccgError):
        B.add_system(plain)                                  # no preconditioner built
    B.close()
    ctx.close()
    plain.close()


@pytest.mark.parametrize("storage", [ib.STORE_FP64, ib.STORE_FP32])
def test_gpu_continuous_batching_equals_solves_alone(storage):
    """Solves admitted while others run (a new one every step, into slots
    freed by retired ones), systems taken out and added again: every result
    is the same bits as the solve alone."""
    probs = [pb.make(pb.poisson2d(s), "piccg", seed=s) for s in (12, 30, 47)]
    probs += [pb.config_abmc_aniso(s, 16, "bfs", seed=s) for s in (9, 14)]
    probs += [pb.config_knn(2500, seed=3, block_size=16)]
    ctxs = [_ctx(P) for P in probs]
    alone = [_alone(c, P.b_run, storage, rr_interval=20) for c, P in zip(ctxs, probs)]
    B = ib.Batch(0)
    B.open(4, storage, rr_interval=20, graph_iters=2)          # fewer slots than requests
    order = [0, 1, 2, 3, 4, 5, 2, 0, 5, 3, 1, 4]
    queue = list(order)
    live = {}                                                    # slot -> (problem index, system index)
    held = {}                                                    # problem index -> [system index, solves]
    done = []
    steps = 0
    while queue or live:
        if queue and len(live) < 4:
            i = queue.pop(0)
            if i not in held:
                held[i] = [B.add_system(ctxs[i]), 0]
            held[i][1] += 1
            live[B.submit(held[i][0], probs[i].b_run, None, 10000, 1e-8)] = (i, held[i][0])
        stopped, running = B.step()
        steps += 1
        assert running <= len(live)
        if stopped:
            xs, res = B.retire(stopped)
            for s, x, r in zip(stopped, xs, res):
                i, k = live.pop(s)
                held[i][1] -= 1
                if held[i][1] == 0:
                    B.remove_system(k)
                    del held[i]
                done.append(i)
                _same((x, r), alone[i])
                assert r.solve_ms > 0
    assert sorted(done) == sorted(order)
    assert steps > len(order)
    # retiring a running or free slot is refused
    k = B.add_system(ctxs[2])
    s = B.submit(k, probs[2].b_run)
    with pytest.raises(ib.IccgError):
        B.retire([s])
    with pytest.raises(ib.IccgError):
        B.remove_system(k)
    while True:
        stopped, _ = B.step()
        if stopped:
            break
    xs, res = B.retire(stopped)
    _same((xs[0], res[0]), alone[2])
    B.close()
    for c in ctxs:
        c.close()
