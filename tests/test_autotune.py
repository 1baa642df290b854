"""Per-matrix tuning logic (iccg_b200.autotune) on the CPU, with fake timers.

The device timings are replaced by functions of the candidate, so the tests
check which candidate the search keeps and what it leaves set, not speed.
"""
import numpy as np

import iccg_b200 as ib
import iccg_b200.autotune as at
import iccg_b200.problems as pb


def test_pick_prefers_fastest_converged():
    trials = [at.Trial("a", 5.0, 10, True), at.Trial("b", 3.0, 10, False), at.Trial("c", 4.0, 12, True)]
    assert at.pick(trials).label == "c"
    none = [at.Trial("a", 5.0, 10, False), at.Trial("b", 3.0, 10, False)]
    assert at.pick(none).label == "b"
    tie = [at.Trial("a", 2.0, 10, True), at.Trial("b", 2.0, 9, True)]
    assert at.pick(tie).label == "a"


def test_tune_ordering_builds_candidates_and_returns_the_fastest():
    A = pb.poisson2d(24)
    cost = {"mc": 7.0, "abmc8": 3.0, "abmc16": 4.0, "abmc32": 9.0, "abmc16_linear": 3.5, "abmc32_linear": 8.0}
    seen = []

    def timer(P):
        seen.append((P.name, P.variant, P.nb, P.nc, P.info.get("blocking")))
        return cost[P.name], 40, True

    P, res = at.tune_ordering(A, timer=timer)
    assert [s[0] for s in seen] == ["mc", "abmc8", "abmc16", "abmc32", "abmc16_linear", "abmc32_linear"]
    assert seen[4][4] == "linear" and seen[1][4] == "bfs"
    assert res.best == "abmc8" and P.name == "abmc8" and P.variant == "abmc"
    assert P.info["block_size"] == 8 and P.nb > 0
    assert len(res.table()) == 6
    # two-element candidates default to breadth-first blocking
    P2, res2 = at.tune_ordering(A, candidates=(("abmc", 16),), timer=timer)
    assert res2.best == "abmc16" and P2.info["blocking"] == "bfs"
    # the chosen problem is the one built: same b, same ordering as make()
    ref = pb.make(A, "abmc", block_size=8, blocking="bfs", seed=0)
    assert np.array_equal(P.new_of_old, ref.new_of_old)
    assert np.array_equal(P.b_run, ref.b_run)


class FakeCtx:
    def __init__(self):
        self.opts = {}
        self.history = []

    def set_option(self, opt, v):
        self.opts[opt] = v
        self.history.append((opt, v))


def test_tune_kernels_coordinate_search_leaves_best_options_set():
    ctx = FakeCtx()
    # cost: the persistent apply faster, per-slice sweeps faster, 112 KB
    # stages best, PDL on better
    def timer():
        o = ctx.opts
        ms = 10.0
        ms -= 2.0 if o[ib.OPT_PERSIST] == 1 else 0.0
        ms -= 1.0 if o[ib.OPT_SWEEP] == 1 else 0.0
        ms -= {0: 0.0, 160: 0.2, 112: 0.5, 80: 0.3}[o[ib.OPT_STAGE_KB]]
        ms -= 0.4 if o[ib.OPT_PDL] == 1 else 0.0
        return ms, 50, True

    res = at.tune_kernels(ctx, np.zeros(4), timer=timer)
    assert ctx.opts == {ib.OPT_PERSIST: 1, ib.OPT_SWEEP: 1, ib.OPT_STAGE_BUFS: 1, ib.OPT_STAGE_KB: 112,
                        ib.OPT_STAGE_ROWS: 256, ib.OPT_PDL: 1, ib.OPT_EARLY: 1, ib.OPT_SPMV_PACK: 1, ib.OPT_SPMV_TPR: 1,
                        ib.OPT_FUSE_UPDATE: 0, ib.OPT_DEFER_X: 0, ib.OPT_UPDATE_CHAIN: 0}
    assert res.choice["persist"] == 1
    assert res.choice["sweep"] == 1 and res.choice["stage_kb"] == 112 and res.choice["pdl"] == 1
    assert abs(res.choice["ms"] - (10.0 - 2.0 - 1.0 - 0.5 - 0.4)) < 1e-12
    assert len(res.trials) == 2 + 2 + 2 + 4 + 3 + 2 + 3 + 2 + 3 + 2 + 2 + 2


def test_tune_kernels_skips_unconverged_settings():
    ctx = FakeCtx()

    def timer():
        # the per-slice kernel "fails" here: fastest but not converged
        if ctx.opts[ib.OPT_SWEEP] == 1:
            return 1.0, 10000, False
        return 5.0, 50, True

    at.tune_kernels(ctx, np.zeros(4), timer=timer)
    assert ctx.opts[ib.OPT_SWEEP] == 0


def test_tune_batch_tunes_one_system_per_class_and_applies_its_choice():
    mats = [pb.poisson2d(18), pb.poisson2d(20), pb.laplace3d_aniso(7, 1.0), pb.poisson2d(40), pb.laplace3d_aniso(8, 1.0)]
    keys = [at.batch_class(A) for A in mats]
    # 2D 5-point: 5 entries per row (rounded); 3D 7-point: 6
    assert keys[0] == keys[1] == (5, 9) and keys[3] == (5, 11)
    assert keys[2] == keys[4] and keys[2][0] == 6
    timed = []

    def timer(P):
        timed.append((P.A.n, P.name))
        # 2D: ABMC 16 wins; 3D: multicolor wins
        best = "abmc16" if P.A.nnz / P.A.n < 6 else "mc"
        return (1.0 if P.name == best else 2.0), 30, True

    probs, rows = at.tune_batch(mats, timer=timer)
    assert len(probs) == len(mats) and len(rows) == 3
    # the largest system of each class is the one timed, once per candidate
    assert sorted({n for n, _ in timed}) == sorted({mats[1].n, mats[3].n, mats[4].n})
    assert len(timed) == 3 * len(at.BATCH_ORDERINGS)
    for A, P, k in zip(mats, probs, keys):
        assert P.A.n == A.n
        assert P.variant == ("abmc" if k[0] < 6 else "piccg")
        if P.variant == "abmc":
            assert P.info["block_size"] == 16
    by = {tuple(r["class"]): r for r in rows}
    assert by[keys[0]]["systems"] == 2 and by[keys[0]]["tuned_on_rows"] == mats[1].n
    assert by[keys[2]]["choice"] == "mc"
    # explicit classes, and their length is checked
    probs2, rows2 = at.tune_batch(mats[:2], classes=["a", "b"], timer=timer)
    assert len(rows2) == 2
    import pytest
    with pytest.raises(ValueError):
        at.tune_batch(mats, classes=["a"], timer=timer)
