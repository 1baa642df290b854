"""GPU parity at the sizes the benchmark measures, against the compiled
reference (oracle/_ref: the reference's own sources built by
oracle/Makefile) and the C restatement.

* The headline system exactly as bench.py builds it: 3D 7-point 128^3
  anisotropic Laplacian, ABMC B=16 with linear blocking (2 colors).
* The 27-point variable-coefficient 96^3 problem, multicolor and ABMC B=8.

On each: SpMV bit for bit against the oracle and the reference, the IC(0)
factor and one preconditioner apply bit for bit against the reference, and
the FP64 solves (fused and plain) to the reference's iteration count +-1 and
||x - x_ref|| / ||x_ref|| <= 1e-10.  The reference's long-double OpenMP
reductions move x with its thread count, so x is compared with its runs at
1, 4 and 16 threads and must lie within 1e-10 of one of them.  The mixed form
(FP32 storage, FP64 recurrences) must reach the true residual and stay within
1e-6 of the FP64 solution.

The device inner product is checked against the exactly rounded dot product
and the reference's long-double dot / nrm2 on ill-conditioned vectors.
"""
import ctypes as C
import math

import numpy as np
import pytest

import iccg_b200 as ib
import iccg_b200.problems as pb
from oracle import bindings as ob
from _util import rel_err

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

X_TOL = 1e-10
THREADS = (1, 4, 16)
need_ref = pytest.mark.skipif(ob.ref() is None, reason="compiled reference not built")


def _ref_problem(P):
    A = P.A
    if P.variant == "piccg":
        return ob.RefProblem(3, A.n, A.rowptr, A.colind, A.val, P.color, P.nc)
    return ob.RefProblem(4, A.n, A.rowptr, A.colind, A.val, P.block_of_old, P.nb, P.block_color, P.nc)


def _ref_solutions(R, P, tol=1e-8):
    out = []
    for t in THREADS:
        ob.ref().ref_set_threads(t)
        x, it, rel, cv, _ = R.cg(P.b_run, np.zeros(P.A_run.n), 10000, tol)
        assert cv
        out.append((t, x, it))
    ob.ref().ref_set_threads(1)
    return out


def _check_system(P):
    R = _ref_problem(P)
    n = P.A_run.n
    # the reference's own A_run, permutation and schedule equal ours
    rp, ci, v = R.arun()
    assert np.array_equal(rp, P.A_run.rowptr) and np.array_equal(ci, P.A_run.colind)
    assert np.array_equal(v, P.A_run.val)
    assert np.array_equal(R.perm(), P.new_of_old)
    ctx = ib.Context(0)
    ctx.upload(P.A_run)
    ctx.set_schedule(P.sched)
    x = ib.gen_uniform(n, 9)
    y = ctx.spmv(x)
    assert np.array_equal(y, ob.spmv(n, P.A_run.rowptr, P.A_run.colind, P.A_run.val, x))
    assert np.array_equal(y, R.spmv(x))
    ctx.build(ib.PRECOND_IC0, 0.0)
    Lx = ctx.export_factor()[2]
    assert np.array_equal(Lx, R.ic0()[2])
    assert np.array_equal(ctx.apply(x), R.apply(x))
    refs = _ref_solutions(R, P)
    for mode in (ib.MODE_FUSED, ib.MODE_PLAIN):
        xs = np.zeros(n)
        res = ctx.solve(P.b_run, xs, 10000, 1e-8, mode=mode, storage=ib.STORE_FP64)
        assert res.converged
        assert min(abs(res.iters - it) for _, _, it in refs) <= 1, (res.iters, [it for _, _, it in refs])
        errs = [rel_err(xs, xr) for _, xr, _ in refs]
        assert min(errs) <= X_TOL, errs
        if mode == ib.MODE_FUSED:
            x64 = xs.copy()
    x32 = np.zeros(n)
    r32 = ctx.solve(P.b_run, x32, 10000, 1e-8, storage=ib.STORE_FP32, rr_interval=50)
    assert r32.converged and r32.true_rel_resid <= 1e-8
    assert rel_err(x32, x64) <= 1e-6
    ctx.close()


@need_ref
def test_bench_system_128_linear_abmc16_matches_reference():
    # bench.py: pb.config_abmc_aniso(128, 16, "linear", seed=0)
    P = pb.config_abmc_aniso(128, 16, "linear", seed=0)
    assert P.A_run.n == 2_097_152 and P.A_run.nnz == 14_581_760 and P.nc == 2
    _check_system(P)


@need_ref
@pytest.mark.parametrize("variant", ["mc", "abmc8"])
def test_diffusion27_96_matches_reference(variant):
    v, B = {"mc": ("piccg", 16), "abmc8": ("abmc", 8)}[variant]
    P = pb.config_diffusion27(96, v, block_size=B, seed=0)
    assert P.A_run.n == 96 ** 3 and P.A_run.nnz == 23_393_656
    _check_system(P)


# ---------------------------------------------------------------------------
# the device inner product
# ---------------------------------------------------------------------------
def _two_product(a, b):
    """Exact products a*b = p + e (Dekker's splitting; no FMA needed)."""
    f = 134217729.0  # 2^27 + 1
    ca, cb = f * a, f * b
    ah = ca - (ca - a)
    al = a - ah
    bh = cb - (cb - b)
    bl = b - bh
    p = a * b
    e = ((ah * bh - p) + ah * bl + al * bh) + al * bl
    return p, e


def _exact_dot(a, b):
    p, e = _two_product(a, b)
    return math.fsum(np.concatenate([p, e]))  # fsum rounds the exact sum once


def _ill_conditioned(n, seed):
    """Half the terms cancel the other half up to a small perturbation, over
    a wide range of magnitudes: sum |a_i b_i| / |a.b| is about 1e8 to 1e12."""
    rng = np.random.default_rng(seed)
    h = n // 2
    u = rng.standard_normal(h) * np.exp2(rng.integers(-20, 21, h))
    v = rng.standard_normal(h) * np.exp2(rng.integers(-20, 21, h))
    w = v * (1.0 + rng.standard_normal(h) * 1e-9)
    a = np.concatenate([u, u, rng.standard_normal(n - 2 * h)])
    b = np.concatenate([v, -w, rng.standard_normal(n - 2 * h)])
    perm = rng.permutation(n)
    return a[perm].copy(), b[perm].copy()


@need_ref
@pytest.mark.parametrize("n", [1000, 65_537, 1_000_000])
def test_device_dot_vs_reference_long_double(n):
    """iccg_dot_dev evaluates in double-double and rounds once: it equals
    the exactly rounded dot product.  The reference's long-double OpenMP
    reduction (cg_crs.cpp:33-50) rounds each partial sum to 64 bits, so it is
    required to agree to within 2 ulp of sum |a_i b_i|, at 1 and 16 threads;
    nrm2 likewise for sqrt(a.a)."""
    torch = pytest.importorskip("torch")
    ctx = ib.Context(0)
    for seed in range(3):
        a, b = _ill_conditioned(n, seed)
        ad = torch.from_numpy(a).cuda()
        bd = torch.from_numpy(b).cuda()
        out = C.c_double(0.0)
        assert ib.lib().iccg_dot_dev(ctx.h, n, C.c_void_p(ad.data_ptr()), C.c_void_p(bd.data_ptr()),
                                     C.byref(out)) == 0
        gpu = out.value
        assert gpu == _exact_dot(a, b)
        scale = float(np.sum(np.abs(a * b)))
        ulp = math.ulp(scale)
        for t in (1, 16):
            ob.ref().ref_set_threads(t)
            ref = ob.ref().ref_dot(n, a.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p))
            assert abs(gpu - ref) <= 2 * ulp, (t, gpu, ref, ulp)
            # nrm2 = sqrt(a.a); the solver's norms are sqrt of the device dot
            assert ib.lib().iccg_dot_dev(ctx.h, n, C.c_void_p(ad.data_ptr()), C.c_void_p(ad.data_ptr()),
                                         C.byref(out)) == 0
            nrm_ref = ob.ref().ref_nrm2(n, a.ctypes.data_as(C.c_void_p))
            nrm_gpu = math.sqrt(out.value)
            assert abs(nrm_gpu - nrm_ref) <= 2 * math.ulp(nrm_ref), (t, nrm_gpu, nrm_ref)
        ob.ref().ref_set_threads(1)
    ctx.close()
