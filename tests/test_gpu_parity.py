"""GPU parity: the CUDA path against the oracle and the golden fixtures.

Bit-exact: SpMV, IC(0) factor, preconditioner apply (all schedules), the
orderings.  FP64 CG (plain and fused): iteration count within 1 of the
reference and ||x - x_ref|| / ||x_ref|| <= 1e-10 (the tolerance of the FP64
path); in practice the fused and plain paths reproduce the reference's
trajectory.  Mixed precision (FP32 storage, FP64 recurrences with residual
replacement): true relative residual <= tol and the error against the FP64
solution is reported.
"""
import numpy as np
import pytest

import iccg_b200 as ib
import iccg_b200.problems as pb
from oracle import bindings as ob
from _util import golden_names, load_golden, golden_sched, to_color_schedule, rel_err

pytestmark = pytest.mark.gpu

X_TOL = 1e-10  # FP64 path: ||x - x_ref|| / ||x_ref||


def _ctx_for(A, sched):
    ctx = ib.Context(0)
    ctx.upload(A)
    ctx.set_schedule(sched)
    return ctx


@pytest.mark.parametrize("name", golden_names())
def test_gpu_matches_golden(name):
    g = load_golden(name)
    n = int(g["n"])
    A = ib.CRS.from_arrays(n, g["run_rowptr"], g["run_colind"], g["run_val"])
    sched = to_color_schedule(golden_sched(g))
    ctx = _ctx_for(A, sched)
    assert np.array_equal(ctx.spmv(g["spmv_x"]), g["spmv_y"])
    kind = {"cg": ib.PRECOND_NONE, "dcg": ib.PRECOND_JACOBI}.get(str(g["variant"]), ib.PRECOND_IC0)
    ctx.build(kind, 0.0)
    if kind == ib.PRECOND_IC0:
        Lp, Li, Lx, Up, Ui, Ux = ctx.export_factor()
        for a, k in ((Lp, "L_rowptr"), (Li, "L_colind"), (Lx, "L_val"), (Up, "LT_colptr"), (Ui, "LT_rowind"),
                     (Ux, "LT_val")):
            assert np.array_equal(a, g[k]), k
    assert np.array_equal(ctx.apply(g["apply_r"]), g["apply_z"])
    for mode in (ib.MODE_PLAIN, ib.MODE_FUSED):
        x = np.zeros(n)
        res = ctx.solve(g["cg_b"], x, 10000, float(g["cg_tol"]), mode=mode)
        assert res.converged == bool(g["cg_converged"])
        assert abs(res.iters - int(g["cg_iters"])) <= 1
        assert rel_err(x, g["cg_x"]) <= X_TOL
    ctx.close()


def _oracle_solve(P, tol=1e-8, kind=2):
    rp, ci, v = P.A_run.rowptr, P.A_run.colind, P.A_run.val
    ic0 = ob.OracleIC0(P.A_run.n, rp, ci, v, 0.0) if kind == 2 else None
    x, it, rel, cv, _ = ob.cg(P.A_run.n, rp, ci, v, P.b_run, np.zeros(P.A_run.n), kind, 10000, tol, ic0, P.sched)
    return ic0, x, it, rel, cv


def _reference_runs(P, tol=1e-8, threads=(1, 2, 4, 8, 16)):
    """x of the compiled reference's ABMC/MC solve for several OpenMP thread
    counts (the long-double reductions combine per-thread partials, so x
    moves with the thread count); empty where the reference was not built."""
    if ob.ref() is None or P.variant not in ("piccg", "abmc"):
        return []
    A = P.A
    if P.variant == "piccg":
        R = ob.RefProblem(3, A.n, A.rowptr, A.colind, A.val, P.color, P.nc)
    else:
        R = ob.RefProblem(4, A.n, A.rowptr, A.colind, A.val, P.block_of_old, P.nb, P.block_color, P.nc)
    out = []
    for t in threads:
        ob.ref().ref_set_threads(t)
        x, it, rel, cv, _ = R.cg(P.b_run, np.zeros(A.n), 10000, tol)
        out.append((t, x, it))
    ob.ref().ref_set_threads(1)
    return out


def _assert_x_parity(x, xo, P):
    """||x - x_ref|| / ||x_ref|| <= 1e-10 against the oracle, or -- on
    ill-conditioned systems where the reference's own OpenMP thread count
    moves x by more than that -- against one of the reference's runs."""
    err = rel_err(x, xo)
    if err <= X_TOL:
        return
    runs = _reference_runs(P)
    assert runs, f"rel err {err:.3e} vs oracle and no compiled reference to compare with"
    best = min(rel_err(x, xr) for _, xr, _ in runs)
    spread = max(rel_err(xr, xo) for _, xr, _ in runs)
    assert best <= X_TOL, (err, best, spread)


@pytest.mark.parametrize("which", ["c1_mc", "abmc64_bfs", "abmc64_lin", "iccg_natural", "d27_abmc", "d27_abmc32",
                                   "d27_abmc64", "abmc_b32", "p2d_abmc64", "d27_mc", "knn"])
def test_gpu_cg_parity_vs_oracle(which):
    if which == "c1_mc":
        P = pb.config_small_mc(128, seed=0)
    elif which == "abmc64_bfs":
        P = pb.config_abmc_aniso(64, 16, "bfs")
    elif which == "abmc64_lin":
        P = pb.config_abmc_aniso(64, 16, "linear")
    elif which == "iccg_natural":
        P = pb.make(pb.laplace3d_aniso(40), "iccg", seed=1)
    elif which == "d27_abmc":
        P = pb.config_diffusion27(40, "abmc", 16)
    elif which == "d27_abmc32":
        # blocks of 32 rows: one group's sweep tile exceeds 48 KB of shared memory
        P = pb.config_diffusion27(32, "abmc", 32)
    elif which == "d27_abmc64":
        P = pb.config_diffusion27(32, "abmc", 64)
    elif which == "abmc_b32":
        # 32-row blocks of a 7-point operator: the staged kernel's batches are single 1024-row groups
        P = pb.config_abmc_aniso(40, 32, "linear")
    elif which == "p2d_abmc64":
        P = pb.make(pb.poisson2d(96), "abmc", block_size=64, blocking="bfs", seed=4)
    elif which == "d27_mc":
        P = pb.config_diffusion27(40, "piccg")
    else:
        P = pb.config_knn(20000, seed=2)
    ic0, xo, ito, relo, cvo = _oracle_solve(P)
    ctx = _ctx_for(P.A_run, P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    # factor and one apply are bit-exact at this size
    Lx = ctx.export_factor()[2]
    assert np.array_equal(Lx, ic0.export()[2])
    r = ib.gen_uniform(P.A_run.n, 11)
    assert np.array_equal(ctx.apply(r), ic0.apply(r, P.sched))
    assert np.array_equal(ctx.spmv(r), ob.spmv(P.A_run.n, P.A_run.rowptr, P.A_run.colind, P.A_run.val, r))
    for mode in (ib.MODE_PLAIN, ib.MODE_FUSED):
        x = np.zeros(P.A_run.n)
        res = ctx.solve(P.b_run, x, 10000, 1e-8, mode=mode)
        assert res.converged and cvo
        assert abs(res.iters - ito) <= 1, (res.iters, ito)
        _assert_x_parity(x, xo, P)
        assert res.true_rel_resid < 1.5e-8
    ctx.close()


@pytest.mark.parametrize("which", ["abmc64", "d27_abmc", "d27_abmc32"])
def test_gpu_mixed_precision(which):
    P = {"abmc64": lambda: pb.config_abmc_aniso(64, 16, "bfs"),
         "d27_abmc": lambda: pb.config_diffusion27(40, "abmc", 16),
         "d27_abmc32": lambda: pb.config_diffusion27(40, "abmc", 32)}[which]()
    ctx = _ctx_for(P.A_run, P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    x64 = np.zeros(P.A_run.n)
    r64 = ctx.solve(P.b_run, x64, 10000, 1e-8, storage=ib.STORE_FP64)
    x32 = np.zeros(P.A_run.n)
    r32 = ctx.solve(P.b_run, x32, 10000, 1e-8, storage=ib.STORE_FP32, rr_interval=50)
    assert r64.converged and r32.converged
    assert r32.true_rel_resid <= 1e-8          # the true residual, in FP64
    assert r32.n_replacements >= 1
    assert rel_err(x32, x64) <= 1e-6           # both are 1e-8-residual solutions
    assert r32.iters <= r64.iters * 1.2 + 5
    ctx.close()


def test_gpu_apply_fp32_close_to_fp64():
    P = pb.config_abmc_aniso(32, 16, "bfs")
    ctx = _ctx_for(P.A_run, P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    r = ib.gen_uniform(P.A_run.n, 3)
    z64 = ctx.apply(r, ib.STORE_FP64)
    z32 = ctx.apply(r, ib.STORE_FP32)
    assert rel_err(z32, z64) < 1e-5
    y64 = ctx.spmv(r, ib.STORE_FP64)
    y32 = ctx.spmv(r, ib.STORE_FP32)
    assert rel_err(y32, y64) < 1e-6
    ctx.close()


def test_gpu_reference_interface():
    """Drop-in use: IC0(A, shift).apply(r, z, sched) and conjugate_gradient()."""
    P = pb.config_small_mc(48, seed=0)
    M = ib.IC0(P.A_run, 0.0, sched=P.sched)
    r = ib.gen_uniform(P.A_run.n, 1)
    z = np.zeros(0)
    M.apply(r, z, P.sched)
    ic0 = ob.OracleIC0(P.A_run.n, P.A_run.rowptr, P.A_run.colind, P.A_run.val, 0.0)
    assert np.array_equal(z, ic0.apply(r, P.sched))
    x = np.zeros(P.A_run.n)
    res = ib.conjugate_gradient(P.A_run, P.b_run, x, M, 10000, 1e-8, P.sched)
    xo, ito, relo, cvo, _ = ob.cg(P.A_run.n, P.A_run.rowptr, P.A_run.colind, P.A_run.val, P.b_run,
                                  np.zeros(P.A_run.n), 2, 10000, 1e-8, ic0, P.sched)
    assert res.converged and abs(res.iters - ito) <= 1 and rel_err(x, xo) <= X_TOL
    for cls, kind in ((ib.Identity, 0), (ib.Jacobi, 1)):
        M2 = cls(P.A_run)
        x2 = np.zeros(P.A_run.n)
        r2 = ib.conjugate_gradient(P.A_run, P.b_run, x2, M2, 10000, 1e-8, None)
        xo2, ito2, _, _, _ = ob.cg(P.A_run.n, P.A_run.rowptr, P.A_run.colind, P.A_run.val, P.b_run,
                                   np.zeros(P.A_run.n), kind, 10000, 1e-8)
        assert abs(r2.iters - ito2) <= 1 and rel_err(x2, xo2) <= X_TOL


# ---------------------------------------------------------------------------
# failure paths (host-side detection; nothing faults the GPU)
# ---------------------------------------------------------------------------
def _indefinite():
    A = pb.poisson2d(12)
    v = A.val.copy()
    for i in range(A.n):
        for k in range(A.rowptr[i], A.rowptr[i + 1]):
            if A.colind[k] == i and i in (37, 90):
                v[k] = -0.5
    return ib.CRS(A.n, A.rowptr, A.colind, v)


def test_gpu_nonpositive_pivot_reported_like_reference():
    A = _indefinite()
    with pytest.raises(ob.OracleError):
        ob.OracleIC0(A.n, A.rowptr, A.colind, A.val, 0.0)
    row = ob.orc().orc_last_error_row()
    ctx = _ctx_for(A, None)
    with pytest.raises(ib.IccgError) as e:
        ctx.build(ib.PRECOND_IC0, 0.0)
    assert e.value.code == ib.ERR_PIVOT_NONPOS
    assert f"row {row}" in str(e.value)
    ctx.build(ib.PRECOND_IC0, 0.0, auto_shift=True)
    assert ctx.shift > 0.0
    z = ctx.apply(np.ones(A.n))
    assert np.all(np.isfinite(z))
    ctx.close()


def test_gpu_missing_diagonal():
    A = ib.CRS.from_arrays(3, [0, 2, 3, 5], [0, 1, 0, 1, 2], [2.0, 1.0, 1.0, 1.0, 3.0])
    ctx = _ctx_for(A, None)
    with pytest.raises(ib.IccgError) as e:
        ctx.build(ib.PRECOND_IC0, 0.0)
    assert e.value.code == ib.ERR_DIAG and "row 1" in str(e.value)
    ctx.close()


def test_gpu_rejects_racy_schedule():
    # an MC schedule of the unpermuted matrix puts dependencies on later colors
    A = pb.poisson2d(8)
    color, nc = ib.color_greedy(A)
    cp = np.zeros(nc + 1, np.int32)
    for c in range(nc):
        cp[c + 1] = cp[c] + np.sum(color == c)
    rows = np.argsort(color[::-1], kind="stable").astype(np.int32)  # any order
    rows = np.concatenate([np.nonzero(color == c)[0] for c in range(nc)]).astype(np.int32)
    bad = ib.ColorSchedule(nc=nc, color_ptr=cp, rows_of_color=rows[::-1].copy())
    ctx = ib.Context(0)
    ctx.upload(A)
    with pytest.raises(ib.IccgError) as e:
        ctx.set_schedule(bad)
    assert e.value.code == ib.ERR_SCHEDULE
    ctx.close()


def test_gpu_failed_schedule_falls_back_to_natural_order():
    # a schedule that fails part-way leaves the context in the natural order,
    # whatever schedule it held before
    A = pb.poisson2d(8)
    color, nc = ib.color_greedy(A)
    cp = np.zeros(nc + 1, np.int32)
    for c in range(nc):
        cp[c + 1] = cp[c] + np.sum(color == c)
    rows = np.concatenate([np.nonzero(color == c)[0] for c in range(nc)]).astype(np.int32)
    bad = ib.ColorSchedule(nc=nc, color_ptr=cp, rows_of_color=rows[::-1].copy())
    r = np.random.default_rng(7).standard_normal(A.n)
    want = ob.OracleIC0(A.n, A.rowptr, A.colind, A.val).apply(r)
    ctx = ib.Context(0)
    ctx.upload(A)
    ctx.build(ib.PRECOND_IC0, 0.0)
    np.testing.assert_array_equal(ctx.apply(r), want)
    with pytest.raises(ib.IccgError):
        ctx.set_schedule(bad)
    ctx.build(ib.PRECOND_IC0, 0.0)
    np.testing.assert_array_equal(ctx.apply(r), want)
    ctx.close()


def test_gpu_state_errors():
    ctx = ib.Context(0)
    with pytest.raises(ib.IccgError) as e:
        ctx.apply(np.ones(3))
    assert e.value.code == ib.ERR_STATE
    ctx.upload(pb.poisson2d(4))
    with pytest.raises(ib.IccgError):
        ctx.apply(np.ones(16))
    ctx.close()


def test_gpu_breakdown_and_maxiter_like_reference():
    A = _indefinite()
    b = np.ones(A.n)
    xo, ito, relo, cvo, _ = ob.cg(A.n, A.rowptr, A.colind, A.val, b, np.zeros(A.n), 0, 10000, 1e-8)
    ctx = _ctx_for(A, None)
    ctx.build(ib.PRECOND_NONE)
    for mode in (ib.MODE_PLAIN, ib.MODE_FUSED):
        x = np.zeros(A.n)
        res = ctx.solve(b, x, 10000, 1e-8, mode=mode)
        assert res.converged == cvo and abs(res.iters - ito) <= 1
    # max_iter cap (cg_crs.cpp:125)
    P = pb.config_small_mc(16)
    ctx2 = _ctx_for(P.A_run, P.sched)
    ctx2.build(ib.PRECOND_IC0, 0.0)
    ic0 = ob.OracleIC0(P.A_run.n, P.A_run.rowptr, P.A_run.colind, P.A_run.val, 0.0)
    for cap in (0, 1, 3):
        xo, ito, relo, cvo, _ = ob.cg(P.A_run.n, P.A_run.rowptr, P.A_run.colind, P.A_run.val, P.b_run,
                                      np.zeros(P.A_run.n), 2, cap, 1e-8, ic0, P.sched)
        for mode in (ib.MODE_PLAIN, ib.MODE_FUSED):
            x = np.zeros(P.A_run.n)
            res = ctx2.solve(P.b_run, x, cap, 1e-8, mode=mode)
            assert res.iters == ito and not res.converged and res.status == "max_iter"
            assert rel_err(x, xo) <= X_TOL if cap else np.all(x == 0)
    ctx.close()
    ctx2.close()


# ---------------------------------------------------------------------------
# full size: size-independent properties at the benchmark configuration
# ---------------------------------------------------------------------------
@pytest.mark.slow
def test_gpu_full_size_abmc_128():
    P = pb.config_abmc_aniso(128, 16, "bfs")
    n = P.A_run.n
    ctx = _ctx_for(P.A_run, P.sched)
    x = ib.gen_uniform(n, 9)
    assert np.array_equal(ctx.spmv(x), ib.host_spmv(P.A_run, x))      # bit-exact at 2.1M rows
    ctx.build(ib.PRECOND_IC0, 0.0)
    ic0 = ob.OracleIC0(n, P.A_run.rowptr, P.A_run.colind, P.A_run.val, 0.0)
    assert np.array_equal(ctx.export_factor()[2], ic0.export()[2])   # factor bit-exact
    assert np.array_equal(ctx.apply(x), ic0.apply(x, P.sched))        # apply bit-exact
    x64 = np.zeros(n)
    r64 = ctx.solve(P.b_run, x64, 10000, 1e-8, storage=ib.STORE_FP64)
    x32 = np.zeros(n)
    r32 = ctx.solve(P.b_run, x32, 10000, 1e-8, storage=ib.STORE_FP32)
    assert r64.converged and r64.true_rel_resid < 1.5e-8
    assert r32.converged and r32.true_rel_resid <= 1e-8
    assert rel_err(x32, x64) < 1e-6
    xs_run = np.empty(n)
    xs_run[P.new_of_old] = P.xstar
    assert rel_err(x64, xs_run) < 1e-4   # error against x* is bounded by cond(A) * 1e-8
    ctx.close()


@pytest.mark.parametrize("which", ["mc2d", "abmc_lin", "abmc_bfs", "d27_abmc8", "d27_abmc32", "d27_mc", "knn_abmc"])
def test_gpu_tiled_kernels_equal_simple_kernels(which):
    """The lane-interleaved kernels (Q order, SELL-32, staged sweeps) give
    the same bits as the one-thread-per-row (per-block) kernels in FP64 --
    apply, SpMV and whole fused solves.  In FP32 storage the lane-interleaved
    backward sweep applies earlier-level entries before in-block ones and
    multiplies by FP32 reciprocal pivots (there is no reference rounding to
    keep there): applies agree to FP32 rounding, solves to the tolerance."""
    P = {"mc2d": lambda: pb.config_small_mc(100, seed=1),
         "abmc_lin": lambda: pb.config_abmc_aniso(40, 16, "linear"),
         "abmc_bfs": lambda: pb.config_abmc_aniso(40, 16, "bfs"),
         "d27_abmc8": lambda: pb.config_diffusion27(24, "abmc", 8),
         "d27_abmc32": lambda: pb.config_diffusion27(24, "abmc", 32),
         "d27_mc": lambda: pb.config_diffusion27(24, "piccg"),
         "knn_abmc": lambda: pb.config_knn(8000, seed=5, block_size=16)}[which]()
    ctx = _ctx_for(P.A_run, P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    r = ib.gen_uniform(P.A_run.n, 21)
    out = {}
    for tiled in (True, False):
        ctx.use_tiled(tiled)
        res = {}
        for st in (ib.STORE_FP64, ib.STORE_FP32):
            x = np.zeros(P.A_run.n)
            rr = ctx.solve(P.b_run, x, 10000, 1e-8, storage=st)
            res[st] = (ctx.apply(r, st), ctx.spmv(r, st), x, rr)
        out[tiled] = res
    a, b = out[True][ib.STORE_FP64], out[False][ib.STORE_FP64]
    for k in range(3):
        assert np.array_equal(a[k], b[k])
    assert a[3].iters == b[3].iters
    a, b = out[True][ib.STORE_FP32], out[False][ib.STORE_FP32]
    assert rel_err(a[0], b[0]) < 1e-5
    assert np.array_equal(a[1], b[1])
    assert a[3].converged and b[3].converged and abs(a[3].iters - b[3].iters) <= 1
    assert a[3].true_rel_resid <= 1e-8 and b[3].true_rel_resid <= 1e-8
    assert rel_err(a[2], b[2]) < 1e-6
    ctx.close()


@pytest.mark.parametrize("which", ["mc2d", "abmc_lin", "abmc_bfs", "d27_abmc8", "d27_abmc16", "d27_abmc32", "abmc_b32",
                                   "p2d_abmc64", "d27_mc", "knn_abmc"])
def test_gpu_staged_sweeps_equal_per_slice_sweeps(which):
    """The staged substitution kernel (double-buffered shared-memory batches)
    against the per-slice two-phase kernel (ICCG_OPT_SWEEP = 1): the same
    bits in FP64 (apply and fused solve, r.z included through the solve);
    in FP32 storage the staged kernel multiplies by reciprocal pivots, so
    applies agree to FP32 rounding and solves to the tolerance."""
    P = {"mc2d": lambda: pb.config_small_mc(100, seed=1),
         "abmc_lin": lambda: pb.config_abmc_aniso(40, 16, "linear"),
         "abmc_bfs": lambda: pb.config_abmc_aniso(40, 16, "bfs"),
         "d27_abmc8": lambda: pb.config_diffusion27(24, "abmc", 8),
         "d27_abmc16": lambda: pb.config_diffusion27(24, "abmc", 16),
         "d27_abmc32": lambda: pb.config_diffusion27(24, "abmc", 32),
         "abmc_b32": lambda: pb.config_abmc_aniso(40, 32, "linear"),
         "p2d_abmc64": lambda: pb.make(pb.poisson2d(96), "abmc", block_size=64, blocking="bfs", seed=4),
         "d27_mc": lambda: pb.config_diffusion27(24, "piccg"),
         "knn_abmc": lambda: pb.config_knn(8000, seed=5, block_size=16)}[which]()
    ctx = _ctx_for(P.A_run, P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    r = ib.gen_uniform(P.A_run.n, 23)
    out = {}
    for opt in (0, 1):
        ctx.set_option(ib.OPT_SWEEP, opt)
        res = {}
        for st in (ib.STORE_FP64, ib.STORE_FP32):
            x = np.zeros(P.A_run.n)
            rr = ctx.solve(P.b_run, x, 10000, 1e-8, storage=st)
            res[st] = (ctx.apply(r, st), x, rr)
        out[opt] = res
    a, b = out[0][ib.STORE_FP64], out[1][ib.STORE_FP64]
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[1], b[1])
    assert a[2].iters == b[2].iters
    a, b = out[0][ib.STORE_FP32], out[1][ib.STORE_FP32]
    assert rel_err(a[0], b[0]) < 1e-5
    assert a[2].converged and b[2].converged and abs(a[2].iters - b[2].iters) <= 2
    assert a[2].true_rel_resid <= 1e-8 and b[2].true_rel_resid <= 1e-8
    assert rel_err(a[1], b[1]) < 1e-6
    ctx.close()


DROPIN = ob.HERE / "_ref" / "dropin_check"


@pytest.mark.skipif(not DROPIN.exists(), reason="drop-in check program not built (needs the reference checkout)")
def test_gpu_dropin_reference_template(tmp_path):
    """The reference's own conjugate_gradient<Precond> (compiled from its
    sources) with iccg::GpuIC0 in place of IC0, files read by the reference's
    readers: same iterations and x as with the reference's IC0."""
    import json
    import subprocess
    A = pb.laplace3d_aniso(20)
    blk, nb = ib.block_partition(A, 16, "bfs")
    bcol, nc = ib.color_blocks(A, blk, nb)
    ib.write_matrix_market(str(tmp_path / "a.mtx"), A, symmetric=True)
    ib.write_assignment_1based(str(tmp_path / "a.blk"), blk, nb)
    ib.write_assignment_1based(str(tmp_path / "a.bcol"), bcol, nc)
    out = subprocess.run([str(DROPIN), str(tmp_path / "a.mtx"), str(tmp_path / "a.blk"), str(tmp_path / "a.bcol"),
                          "1e-8"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    d = json.loads(out.stdout.strip().splitlines()[-1])
    assert abs(d["adapter_iters"] - d["ref_iters"]) <= 1
    assert d["adapter_x_rel_err"] <= X_TOL
    assert d["gpu_converged"] == 1 and abs(d["gpu_iters"] - d["ref_iters"]) <= 1
    assert d["gpu_x_rel_err"] <= X_TOL


@pytest.mark.parametrize("which", ["abmc_lin", "d27_mc"])
def test_gpu_pdl_launches_give_the_same_bits(which):
    """Programmatic dependent launch only lets a kernel's CTAs be placed
    early; every kernel still waits for its predecessor.  FP64 and FP32
    solves and applies must be identical with it on and off."""
    P = {"abmc_lin": lambda: pb.config_abmc_aniso(40, 16, "linear"),
         "d27_mc": lambda: pb.config_diffusion27(24, "piccg")}[which]()
    ctx = _ctx_for(P.A_run, P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    r = ib.gen_uniform(P.A_run.n, 29)
    out = {}
    for pdl in (1, 0):
        ctx.set_option(ib.OPT_PDL, pdl)
        res = []
        for st in (ib.STORE_FP64, ib.STORE_FP32):
            x = np.zeros(P.A_run.n)
            rr = ctx.solve(P.b_run, x, 10000, 1e-8, storage=st)
            res.append((ctx.apply(r, st), x, rr.iters))
        out[pdl] = res
    for a, b in zip(out[1], out[0]):
        assert np.array_equal(a[0], b[0])
        assert np.array_equal(a[1], b[1])
        assert a[2] == b[2]
    ctx.close()


@pytest.mark.parametrize("which", ["abmc_lin", "abmc_bfs", "d27_mc", "mc2d"])
def test_gpu_early_loads_give_the_same_bits(which):
    """Loads before the wait on the previous launch (ICCG_OPT_EARLY) only
    move reads of data that launch cannot write ahead of the wait: solves
    (FP64 and mixed, with the fused update and deferred x as well) and
    applies are identical with them off, on for FP32 storage (the default)
    and on for both storages, over several solves in a row."""
    P = {"abmc_lin": lambda: pb.config_abmc_aniso(40, 16, "linear"),
         "abmc_bfs": lambda: pb.config_abmc_aniso(40, 16, "bfs"),
         "d27_mc": lambda: pb.config_diffusion27(24, "piccg"),
         "mc2d": lambda: pb.config_small_mc(100, seed=1)}[which]()
    ctx = _ctx_for(P.A_run, P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    r = ib.gen_uniform(P.A_run.n, 37)
    out = {}
    for early in (0, 1, 3):
        ctx.set_option(ib.OPT_EARLY, early)
        res = []
        for opt in (None, ib.OPT_FUSE_UPDATE, ib.OPT_DEFER_X):
            if opt is not None:
                ctx.set_option(opt, 1)
            for st, cap, rri in ((ib.STORE_FP64, 10000, 50), (ib.STORE_FP32, 10000, 50), (ib.STORE_FP32, 10000, 7),
                                 (ib.STORE_FP64, 9, 50)):
                for _ in range(2):
                    x = np.zeros(P.A_run.n)
                    rr = ctx.solve(P.b_run, x, cap, 1e-8, storage=st, rr_interval=rri)
                    res.append((x, rr.iters, rr.status, rr.n_replacements))
            if opt is not None:
                ctx.set_option(opt, 0)
        for st in (ib.STORE_FP64, ib.STORE_FP32):
            res.append((ctx.apply(r, st), 0, "", 0))
        out[early] = res
    ctx.set_option(ib.OPT_EARLY, 1)
    for e in (1, 3):
        for a, b in zip(out[e], out[0]):
            assert np.array_equal(a[0], b[0])
            assert a[1:] == b[1:]
    ctx.close()


@pytest.mark.parametrize("which", ["abmc_lin", "abmc_bfs", "d27_mc", "mc2d", "knn_abmc"])
def test_gpu_update_chain_gives_the_same_bits(which):
    """The update with the first (chain-only) forward level in its launch
    (ICCG_OPT_UPDATE_CHAIN) does each element's fused multiply-adds of the
    update and the chain-only sweep: solves keep their bits, iterations and
    statuses in FP64 and mixed storage, with replacement, iteration caps and
    early loads on and off.  (Systems whose first level is not chain-only
    take the usual path.)"""
    P = {"abmc_lin": lambda: pb.config_abmc_aniso(40, 16, "linear"),
         "abmc_bfs": lambda: pb.config_abmc_aniso(40, 16, "bfs"),
         "d27_mc": lambda: pb.config_diffusion27(24, "piccg"),
         "mc2d": lambda: pb.config_small_mc(100, seed=1),
         "knn_abmc": lambda: pb.config_knn(8000, seed=5, block_size=16)}[which]()
    ctx = _ctx_for(P.A_run, P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    out = {}
    for uc in (1, 0):
        ctx.set_option(ib.OPT_UPDATE_CHAIN, uc)
        res = []
        for early in (1, 3):
            ctx.set_option(ib.OPT_EARLY, early)
            for st, cap, rri in ((ib.STORE_FP64, 10000, 50), (ib.STORE_FP32, 10000, 50), (ib.STORE_FP32, 10000, 7),
                                 (ib.STORE_FP64, 9, 50)):
                x = np.zeros(P.A_run.n)
                rr = ctx.solve(P.b_run, x, cap, 1e-8, storage=st, rr_interval=rri)
                res.append((x, rr.iters, rr.status, rr.n_replacements, rr.true_rel_resid))
        out[uc] = res
    ctx.set_option(ib.OPT_UPDATE_CHAIN, 0)
    ctx.set_option(ib.OPT_EARLY, 1)
    for a, b in zip(out[1], out[0]):
        assert np.array_equal(a[0], b[0])
        assert a[1:] == b[1:]
    ctx.close()


@pytest.mark.parametrize("which", ["abmc_lin", "d27_mc", "d27_abmc8"])
def test_gpu_stage_budget_keeps_fp64_bits(which):
    """The staged kernel's batch budget (ICCG_OPT_STAGE_KB) only changes how
    many groups a CTA stages at once, and which levels fall back to the
    per-slice kernel: FP64 applies and solves keep their bits; FP32 storage
    (reciprocal pivots on the staged kernel, division on the per-slice one)
    agrees to FP32 rounding and converges to the tolerance."""
    P = {"abmc_lin": lambda: pb.config_abmc_aniso(40, 16, "linear"),
         "d27_mc": lambda: pb.config_diffusion27(24, "piccg"),
         "d27_abmc8": lambda: pb.config_diffusion27(24, "abmc", 8)}[which]()
    ctx = _ctx_for(P.A_run, P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    r = ib.gen_uniform(P.A_run.n, 31)
    out = {}
    plans = {}
    for kb in (0, 48, 4):
        ctx.set_option(ib.OPT_STAGE_KB, kb)
        plans[kb] = [k for k, _ in ctx.sweep_plan(ib.STORE_FP32, True)]
        res = {}
        for st in (ib.STORE_FP64, ib.STORE_FP32):
            x = np.zeros(P.A_run.n)
            rr = ctx.solve(P.b_run, x, 10000, 1e-8, storage=st)
            res[st] = (ctx.apply(r, st), x, rr)
        out[kb] = res
    ctx.set_option(ib.OPT_STAGE_KB, 0)
    assert all(k in ("chain", "staged") for k in plans[0]), plans[0]
    if which != "abmc_lin":
        assert "two_phase" in plans[4], plans[4]   # single groups that exceed 4 KB
    for kb in (48, 4):
        a, b = out[0][ib.STORE_FP64], out[kb][ib.STORE_FP64]
        assert np.array_equal(a[0], b[0])
        assert np.array_equal(a[1], b[1])
        assert a[2].iters == b[2].iters
        a, b = out[0][ib.STORE_FP32], out[kb][ib.STORE_FP32]
        assert rel_err(a[0], b[0]) < 1e-5
        assert a[2].converged and b[2].converged and abs(a[2].iters - b[2].iters) <= 2
        assert b[2].true_rel_resid <= 1e-8
    ctx.close()


def test_gpu_sweep_plan_reports_kernels():
    """Units of 32 rows on the 27-point operator: one group's stage needs
    more than half the shared memory, so the levels where it fits one buffer
    run the staged kernel single-buffered (FP32, and the FP64 forward sweep
    where FP64 values fit too) and the others the per-slice two-phase kernel;
    the exact-order FP64 backward sweep stays per-slice; the untiled path
    reports the CSR kernels."""
    P = pb.config_diffusion27(24, "abmc", 32)
    ctx = _ctx_for(P.A_run, P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    for st in (ib.STORE_FP64, ib.STORE_FP32):
        for fwd in (True, False):
            plan = ctx.sweep_plan(st, fwd)
            assert len(plan) == P.nc
            assert all(k in ("two_phase", "staged", "chain") and g >= 1 for k, g in plan), plan
            if st == ib.STORE_FP64 and not fwd:
                assert all(k != "staged" for k, _ in plan), plan
    assert any(k == "staged" for k, _ in ctx.sweep_plan(ib.STORE_FP32, True))
    ctx.use_tiled(False)
    assert all(k == "csr" for k, _ in ctx.sweep_plan(ib.STORE_FP64, True))
    ctx.use_tiled(True)
    ctx.close()


@pytest.mark.parametrize("which", ["abmc_lin32", "d27_mc", "d27_abmc8"])
def test_gpu_single_buffered_staging_gives_the_same_bits(which):
    """The staged kernel with one shared-memory buffer per CTA, refilled after
    each batch (ICCG_OPT_STAGE_BUFS 1, the default), and with two (the next
    batch copied while the current one is worked on): only when a batch's
    copy is issued changes, so applies and solves are identical in both
    storages."""
    P = {"abmc_lin32": lambda: pb.config_abmc_aniso(32, 16, "linear"),
         "d27_mc": lambda: pb.config_diffusion27(24, "piccg"),
         "d27_abmc8": lambda: pb.config_diffusion27(24, "abmc", 8)}[which]()
    ctx = _ctx_for(P.A_run, P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    r = ib.gen_uniform(P.A_run.n, 43)
    out = {}
    for bufs in (2, 1):
        ctx.set_option(ib.OPT_STAGE_BUFS, bufs)
        res = []
        for st in (ib.STORE_FP64, ib.STORE_FP32):
            x = np.zeros(P.A_run.n)
            rr = ctx.solve(P.b_run, x, 10000, 1e-8, storage=st)
            res.append((ctx.apply(r, st), x, rr.iters))
        out[bufs] = res
    ctx.set_option(ib.OPT_STAGE_BUFS, 1)
    assert any(k == "staged" for k, _ in ctx.sweep_plan(ib.STORE_FP32, True))
    for a, b in zip(out[2], out[1]):
        assert np.array_equal(a[0], b[0])
        assert np.array_equal(a[1], b[1])
        assert a[2] == b[2]
    ctx.close()


def _dense_crs(rows):
    d = np.asarray(rows, dtype=float)
    n = d.shape[0]
    rp, ci, v = [0], [], []
    for i in range(n):
        for j in range(n):
            if d[i, j] != 0.0:
                ci.append(j)
                v.append(d[i, j])
        rp.append(len(ci))
    return ib.CRS.from_arrays(n, np.array(rp, np.int32), np.array(ci, np.int32), np.array(v))


@pytest.mark.parametrize("which", ["n1_mc", "n2_mc", "n2_abmc", "p2d_3_mc", "l3d_3_abmc16", "l3d_3_abmc4_lin",
                                   "natural_33", "knn_40"])
def test_gpu_tiny_and_ragged_systems_match_oracle(which):
    """Systems far below one 32-row slice or with ragged units: a 1x1 and a
    2x2 matrix, 9 and 27 rows (one partial slice; 16-row blocks of which the
    last is cut short; 4-row linear blocks), 33 rows in natural order (one
    full slice and one row) and a 40-point k-NN graph.  Factor, apply and
    SpMV bit for bit, FP64 CG on both paths as the oracle's, and the mixed
    form to the true residual."""
    P = {"n1_mc": lambda: pb.make(_dense_crs([[4.0]]), "piccg", seed=1),
         "n2_mc": lambda: pb.make(_dense_crs([[2.0, -1.0], [-1.0, 2.0]]), "piccg", seed=2),
         "n2_abmc": lambda: pb.make(_dense_crs([[2.0, -1.0], [-1.0, 2.0]]), "abmc", block_size=16, seed=2),
         "p2d_3_mc": lambda: pb.make(pb.poisson2d(3), "piccg", seed=3),
         "l3d_3_abmc16": lambda: pb.make(pb.laplace3d_aniso(3), "abmc", block_size=16, seed=4),
         "l3d_3_abmc4_lin": lambda: pb.make(pb.laplace3d_aniso(3), "abmc", block_size=4, blocking="linear", seed=5),
         "natural_33": lambda: pb.make(ib.gen_stencil_2d5(33, 1), "iccg", seed=6),
         "knn_40": lambda: pb.config_knn(40, seed=7, block_size=16)}[which]()
    ic0, xo, ito, relo, cvo = _oracle_solve(P)
    ctx = _ctx_for(P.A_run, P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    assert np.array_equal(ctx.export_factor()[2], ic0.export()[2])
    r = ib.gen_uniform(P.A_run.n, 13)
    assert np.array_equal(ctx.apply(r), ic0.apply(r, P.sched))
    A = P.A_run
    assert np.array_equal(ctx.spmv(r), ob.spmv(A.n, A.rowptr, A.colind, A.val, r))
    for mode in (ib.MODE_PLAIN, ib.MODE_FUSED):
        x = np.zeros(A.n)
        res = ctx.solve(P.b_run, x, 10000, 1e-8, mode=mode)
        assert res.converged and cvo
        assert abs(res.iters - ito) <= 1, (res.iters, ito)
        _assert_x_parity(x, xo, P)
    x = np.zeros(A.n)
    res = ctx.solve(P.b_run, x, 10000, 1e-8, storage=ib.STORE_FP32)
    assert res.converged and res.true_rel_resid <= 1e-8
    ctx.close()


@pytest.mark.parametrize("tiled", [False, True])
def test_gpu_solve_dev_on_alternating_buffer_pairs(tiled):
    """solve_dev straight on caller buffers (the untiled path passes b and x
    to the captured iteration graphs as they are): alternating between two
    (b, x) pairs must re-record the graphs for each pair, so every solve
    writes its own x and matches the oracle's."""
    torch = pytest.importorskip("torch")
    P = pb.config_abmc_aniso(24, 16, "bfs", seed=0)
    n = P.A_run.n
    ic0, xo, ito, relo, cvo = _oracle_solve(P)
    b2 = ib.gen_uniform(n, 77)
    ic0b = ob.OracleIC0(n, P.A_run.rowptr, P.A_run.colind, P.A_run.val, 0.0)
    xo2, ito2, _, _, _ = ob.cg(n, P.A_run.rowptr, P.A_run.colind, P.A_run.val, b2, np.zeros(n), 2, 10000, 1e-8,
                               ic0b, P.sched)
    ctx = _ctx_for(P.A_run, P.sched)
    ctx.use_tiled(tiled)
    ctx.build(ib.PRECOND_IC0, 0.0)
    pairs = [(torch.from_numpy(P.b_run).cuda(), torch.zeros(n, dtype=torch.float64, device="cuda"), xo, ito),
             (torch.from_numpy(b2).cuda(), torch.zeros(n, dtype=torch.float64, device="cuda"), xo2, ito2)]
    for k in (0, 1, 0, 1):
        bd, xd, want, it = pairs[k]
        xd.zero_()
        torch.cuda.synchronize()
        res = ctx.solve_dev(bd.data_ptr(), xd.data_ptr(), 10000, 1e-8)
        assert res.converged and abs(res.iters - it) <= 1
        assert rel_err(xd.cpu().numpy(), want) <= X_TOL
        # the other pair's x holds its own solution (or zeros), never this one
        other = pairs[1 - k][1].cpu().numpy()
        assert not other.any() or rel_err(other, want) > 1e-3
    ctx.close()


@pytest.mark.parametrize("which", ["abmc_lin", "abmc_bfs", "d27_mc", "d27_abmc8", "mc2d", "knn_abmc"])
def test_gpu_fused_update_gives_the_same_bits(which):
    """The CG update done inside the forward sweep's launches
    (ICCG_OPT_FUSE_UPDATE) against the update kernel on its own:
    the same arithmetic per row, so FP64 solves keep their bits and
    iteration counts; FP32 storage converges to the true residual."""
    P = {"abmc_lin": lambda: pb.config_abmc_aniso(40, 16, "linear"),
         "abmc_bfs": lambda: pb.config_abmc_aniso(40, 16, "bfs"),
         "d27_mc": lambda: pb.config_diffusion27(24, "piccg"),
         "d27_abmc8": lambda: pb.config_diffusion27(24, "abmc", 8),
         "mc2d": lambda: pb.config_small_mc(100, seed=1),
         "knn_abmc": lambda: pb.config_knn(8000, seed=5, block_size=16)}[which]()
    ctx = _ctx_for(P.A_run, P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    out = {}
    for fuse in (1, 0):
        ctx.set_option(ib.OPT_FUSE_UPDATE, fuse)
        res = []
        for st in (ib.STORE_FP64, ib.STORE_FP32):
            x = np.zeros(P.A_run.n)
            rr = ctx.solve(P.b_run, x, 10000, 1e-8, storage=st)
            res.append((x, rr))
        out[fuse] = res
    (xa, ra), (xb, rb) = out[1][0], out[0][0]
    assert ra.converged and ra.iters == rb.iters and np.array_equal(xa, xb)
    (xa, ra), (xb, rb) = out[1][1], out[0][1]
    assert ra.converged and ra.true_rel_resid <= 1e-8 and abs(ra.iters - rb.iters) <= 1
    assert rel_err(xa, xb) < 1e-6
    ctx.close()


@pytest.mark.parametrize("which", ["abmc_lin", "d27_mc", "mc2d"])
def test_gpu_deferred_x_update_gives_the_same_bits(which):
    """x += alpha p done by the p update (ICCG_OPT_DEFER_X) against the r
    update doing it (the default): the same bits for converged solves (the
    last x update left pending and applied before the true residual), for
    iteration caps (stops at the p update), in FP64 and in the mixed form
    (whose FP64 confirmation resumes a stopped solve)."""
    P = {"abmc_lin": lambda: pb.config_abmc_aniso(40, 16, "linear"),
         "d27_mc": lambda: pb.config_diffusion27(24, "piccg"),
         "mc2d": lambda: pb.config_small_mc(100, seed=1)}[which]()
    ctx = _ctx_for(P.A_run, P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    out = {}
    for dx in (1, 0):
        ctx.set_option(ib.OPT_DEFER_X, dx)
        res = []
        for st, cap, tol, rri, gi in ((ib.STORE_FP64, 10000, 1e-8, 50, 8), (ib.STORE_FP64, 7, 1e-8, 50, 8),
                                      (ib.STORE_FP64, 10000, 1e-3, 50, 3), (ib.STORE_FP32, 10000, 1e-8, 50, 8),
                                      (ib.STORE_FP32, 10000, 1e-8, 7, 5), (ib.STORE_FP32, 9, 1e-8, 4, 8)):
            x = np.zeros(P.A_run.n)
            r = ctx.solve(P.b_run, x, cap, tol, storage=st, rr_interval=rri, graph_iters=gi)
            res.append((x, r))
        out[dx] = res
    ctx.set_option(ib.OPT_DEFER_X, 0)
    for (xa, ra), (xb, rb) in zip(out[1], out[0]):
        assert ra.iters == rb.iters and ra.status == rb.status and ra.n_replacements == rb.n_replacements
        assert np.array_equal(xa, xb)
        assert ra.true_rel_resid == rb.true_rel_resid
    assert out[1][1][1].status == "max_iter" and out[1][0][1].converged
    ctx.close()


@pytest.mark.parametrize("which", ["abmc_lin", "d27_abmc8", "knn_abmc"])
def test_gpu_packed_spmv_gives_the_same_bits(which):
    """The FP32 SpMV reading (value, column) words (ICCG_OPT_SPMV_PACK, the
    default) against two separate loads: the same bits for the product and
    for a mixed-precision solve."""
    P = {"abmc_lin": lambda: pb.config_abmc_aniso(40, 16, "linear"),
         "d27_abmc8": lambda: pb.config_diffusion27(24, "abmc", 8),
         "knn_abmc": lambda: pb.config_knn(8000, seed=5, block_size=16)}[which]()
    ctx = _ctx_for(P.A_run, P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    v = ib.gen_uniform(P.A_run.n, 41)
    out = {}
    for pk in (1, 0):
        ctx.set_option(ib.OPT_SPMV_PACK, pk)
        x = np.zeros(P.A_run.n)
        r = ctx.solve(P.b_run, x, 10000, 1e-8, storage=ib.STORE_FP32)
        out[pk] = (ctx.spmv(v, ib.STORE_FP32), x, r)
    ctx.set_option(ib.OPT_SPMV_PACK, 1)
    assert np.array_equal(out[1][0], out[0][0])
    assert np.array_equal(out[1][1], out[0][1]) and out[1][2].iters == out[0][2].iters
    ctx.close()


@pytest.mark.parametrize("which", ["abmc_lin", "d27_mc"])
def test_gpu_stage_rows_give_the_same_bits(which):
    """Staged batches of 256 to 2048 rows (ICCG_OPT_STAGE_ROWS): how rows are
    grouped into CTAs changes, the arithmetic of every row does not."""
    P = {"abmc_lin": lambda: pb.config_abmc_aniso(40, 16, "linear"),
         "d27_mc": lambda: pb.config_diffusion27(24, "piccg")}[which]()
    ctx = _ctx_for(P.A_run, P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    r = ib.gen_uniform(P.A_run.n, 47)
    out = {}
    for rows in (256, 512, 128, 1024, 2048):
        ctx.set_option(ib.OPT_STAGE_ROWS, rows)
        res = []
        for st in (ib.STORE_FP64, ib.STORE_FP32):
            x = np.zeros(P.A_run.n)
            rr = ctx.solve(P.b_run, x, 10000, 1e-8, storage=st)
            res.append((ctx.apply(r, st), x, rr.iters))
        out[rows] = res
    ctx.set_option(ib.OPT_STAGE_ROWS, 256)
    for rows in (512, 128, 1024, 2048):
        for a, b in zip(out[rows], out[256]):
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]
    ctx.close()


@pytest.mark.parametrize("which", ["d27_mc", "knn_abmc", "abmc_lin"])
def test_gpu_spmv_threads_per_row(which):
    """The FP32 SpMV with 2 or 4 threads per row (ICCG_OPT_SPMV_TPR): the
    product within FP32-storage rounding of the FP64 one, deterministic from
    run to run, mixed solves to the true residual; FP64 storage keeps one
    thread per row and its bits."""
    P = {"d27_mc": lambda: pb.config_diffusion27(24, "piccg"),
         "knn_abmc": lambda: pb.config_knn(8000, seed=5, block_size=16),
         "abmc_lin": lambda: pb.config_abmc_aniso(40, 16, "linear")}[which]()
    ctx = _ctx_for(P.A_run, P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    v = ib.gen_uniform(P.A_run.n, 53)
    y64 = ctx.spmv(v, ib.STORE_FP64)
    x64 = np.zeros(P.A_run.n)
    r64 = ctx.solve(P.b_run, x64, 10000, 1e-8, storage=ib.STORE_FP64)
    for tpr in (2, 4, 1):
        ctx.set_option(ib.OPT_SPMV_TPR, tpr)
        y = ctx.spmv(v, ib.STORE_FP32)
        assert np.array_equal(y, ctx.spmv(v, ib.STORE_FP32))
        assert rel_err(y, y64) < 1e-6
        assert np.array_equal(ctx.spmv(v, ib.STORE_FP64), y64)
        x = np.zeros(P.A_run.n)
        r = ctx.solve(P.b_run, x, 10000, 1e-8, storage=ib.STORE_FP32)
        assert r.converged and r.true_rel_resid <= 1e-8
        # the mixed form's distance to the FP64 solution (conditioning x tol)
        assert rel_err(x, x64) < 1e-5
        x2 = np.zeros(P.A_run.n)
        r2 = ctx.solve(P.b_run, x2, 10000, 1e-8, storage=ib.STORE_FP64)
        assert r2.iters == r64.iters and np.array_equal(x2, x64)
    ctx.close()
