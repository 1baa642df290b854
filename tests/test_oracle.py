"""The oracle (C restatement) pinned against the reference.

1. Against the committed golden fixtures (outputs of the compiled reference,
   tests/golden/make_golden.py): bit-exact orderings, factor, apply, spmv and
   the whole CG trajectory (iteration count, residual, x).
2. Against the compiled reference itself (oracle/_ref) where it was built:
   more sizes, multi-threaded OpenMP runs, the file readers and their errors.
"""
import numpy as np
import pytest

from oracle import bindings as ob
from _util import golden_names, load_golden, golden_sched

NAMES = golden_names()


def test_fixtures_present():
    assert len(NAMES) >= 10


@pytest.mark.parametrize("name", NAMES)
def test_restatement_matches_golden(name):
    g = load_golden(name)
    n = int(g["n"])
    v = str(g["variant"])
    rp, ci, vals = g["A_rowptr"], g["A_colind"], g["A_val"]
    sched = golden_sched(g)
    # main() set-up: permutation, P^T A P, expansion, schedule
    if v in ("piccg", "abmc"):
        if v == "piccg":
            perm = ob.perm_by_color(g["color"])
        else:
            perm = ob.perm_by_block_color(g["block_of_old"], g["block_color"])
        assert np.array_equal(perm, g["perm"])
        lrp, lci, lv = ob.ptap_lower(n, rp, ci, vals, perm)
        frp, fci, fv = ob.expand_lower_to_full(n, lrp, lci, lv)
        assert np.array_equal(frp, g["run_rowptr"]) and np.array_equal(fci, g["run_colind"])
        assert np.array_equal(fv, g["run_val"])
        if v == "piccg":
            color = g["color"]
            cp, rc = ob.color_schedule(color, int(g["nc"]), perm)
            assert np.array_equal(cp, g["color_ptr"]) and np.array_equal(rc, g["rows_of_color"])
        else:
            cpb, boc, bp, rob = ob.abmc_schedule(perm, g["block_of_old"], g["block_color"], int(g["nb"]), int(g["nc"]))
            for a, b in ((cpb, "color_ptr_blk"), (boc, "blocks_of_color"), (bp, "block_ptr"), (rob, "rows_of_block")):
                assert np.array_equal(a, g[b]), b
    else:
        frp, fci, fv = rp, ci, vals
        assert np.array_equal(g["run_val"], vals)
    # spmv
    y = ob.spmv(n, frp, fci, fv, g["spmv_x"])
    assert np.array_equal(y, g["spmv_y"])
    # preconditioner
    kind = {"cg": 0, "dcg": 1}.get(v, 2)
    ic0 = None
    if kind == 2:
        ic0 = ob.OracleIC0(n, frp, fci, fv, 0.0)
        for a, key in zip(ic0.export(), ("L_rowptr", "L_colind", "L_val", "LT_colptr", "LT_rowind", "LT_val")):
            assert np.array_equal(a, g[key]), key
        z = ic0.apply(g["apply_r"], sched)
        assert np.array_equal(z, g["apply_z"])
    # the whole solve
    x, it, rel, cv, _ = ob.cg(n, frp, fci, fv, g["cg_b"], np.zeros(n), kind, 10000, float(g["cg_tol"]), ic0, sched)
    assert it == int(g["cg_iters"])
    assert rel == float(g["cg_rel"])
    assert cv == bool(g["cg_converged"])
    assert np.array_equal(x, g["cg_x"])


def test_saad_iteration_counts():
    # the reference's own smoke matrix with b = 1, tol 1e-8 (cg_crs.cpp:439-440)
    got = {name.split("_")[1]: int(load_golden(name)["cg_iters"]) for name in NAMES if name.startswith("saad_")}
    assert got == {"cg": 10, "dcg": 10, "iccg": 5, "piccg": 5, "abmc": 5}


# ---------------------------------------------------------------------------
# against the compiled reference
# ---------------------------------------------------------------------------
needs_ref = pytest.mark.skipif(ob.REF_SO.exists() is False, reason="compiled reference not built here")


def _problem(kind):
    import iccg_b200.problems as pb
    if kind == "2d":
        return pb.make(pb.poisson2d(40), "piccg", seed=1)
    if kind == "3d_bfs":
        return pb.make(pb.laplace3d_aniso(14), "abmc", block_size=16, blocking="bfs", seed=2)
    if kind == "3d_lin":
        return pb.make(pb.laplace3d_aniso(14), "abmc", block_size=16, blocking="linear", seed=3)
    if kind == "27":
        import iccg_b200 as ib
        return pb.make(ib.gen_diffusion27(10, 9, 8, 1e4, 5), "abmc", block_size=8, seed=5)
    if kind == "knn":
        return pb.config_knn(3000, seed=4)
    raise KeyError(kind)


@needs_ref
@pytest.mark.parametrize("kind", ["2d", "3d_bfs", "3d_lin", "27", "knn"])
@pytest.mark.parametrize("threads", [1, 4])
def test_restatement_matches_reference(kind, threads):
    P = _problem(kind)
    A = P.A
    ob.ref().ref_set_threads(threads)
    try:
        if P.variant == "piccg":
            R = ob.RefProblem(3, A.n, A.rowptr, A.colind, A.val, P.color, P.nc)
        else:
            R = ob.RefProblem(4, A.n, A.rowptr, A.colind, A.val, P.block_of_old, P.nb, P.block_color, P.nc)
        rp, ci, v = R.arun()
        perm = R.perm()
        if P.variant == "piccg":
            assert np.array_equal(perm, ob.perm_by_color(P.color))
        else:
            assert np.array_equal(perm, ob.perm_by_block_color(P.block_of_old, P.block_color))
        ic0 = ob.OracleIC0(A.n, rp, ci, v, 0.0)
        for a, b in zip(ic0.export(), R.ic0()):
            assert np.array_equal(a, b)
        r = np.random.default_rng(0).uniform(-1, 1, A.n)
        assert np.array_equal(ic0.apply(r, P.sched), R.apply(r))
        assert np.array_equal(ob.spmv(A.n, rp, ci, v, r), R.spmv(r))
        xr, itr, relr, cvr, _ = R.cg(P.b_run, np.zeros(A.n), 10000, 1e-8)
        xo, ito, relo, cvo, _ = ob.cg(A.n, rp, ci, v, P.b_run, np.zeros(A.n), 2, 10000, 1e-8, ic0, P.sched)
        assert cvr and cvo
        if threads == 1:
            assert itr == ito and relr == relo and np.array_equal(xr, xo)
        else:
            # OpenMP partial sums of the long-double reductions combine in a
            # thread-dependent order: same iterations, x to rounding level
            assert abs(itr - ito) <= 1
            assert np.linalg.norm(xr - xo) <= 1e-12 * np.linalg.norm(xr)
    finally:
        ob.ref().ref_set_threads(1)


@needs_ref
def test_dot_nrm2_match_reference():
    rng = np.random.default_rng(3)
    ob.ref().ref_set_threads(1)
    for n in (1, 7, 1000, 100003):
        a, b = rng.standard_normal(n), rng.standard_normal(n)
        assert ob.dot(a, b) == ob.ref().ref_dot(n, a.ctypes.data, b.ctypes.data)
        assert ob.nrm2(a) == ob.ref().ref_nrm2(n, a.ctypes.data)


@needs_ref
def test_readers_match_reference(tmp_path):
    import iccg_b200 as ib
    A = ib.gen_stencil_2d5(7, 5)
    p = tmp_path / "a.mtx"
    ib.write_matrix_market(str(p), A, symmetric=True)
    n, rp, ci, v = ob.read_mm(p)
    n2, rp2, ci2, v2 = ob.ref_read_mm(p)
    assert n == n2 and np.array_equal(rp, rp2) and np.array_equal(ci, ci2) and np.array_equal(v, v2)
    col = tmp_path / "a.col"
    col.write_text("3\n" + "".join(f"{i + 1} {(i % 3) + 1}\n" for i in range(n)))
    c1, k1 = ob.read_assignment(col, n)
    c2, k2 = ob.ref_read_assignment(0, col, n)
    assert k1 == k2 == 3 and np.array_equal(c1, c2)


@needs_ref
@pytest.mark.parametrize("text", [
    "3\n1 1\n2 2\n",            # not every node assigned
    "0\n1 1\n",                 # non-positive count
    "2\n1 3\n2 1\n3 1\n",       # value out of range
    "2\n0 1\n",                 # id out of range
])
def test_assignment_errors_match_reference(tmp_path, text):
    p = tmp_path / "bad.col"
    p.write_text(text)
    with pytest.raises(ob.OracleError):
        ob.read_assignment(p, 3)
    with pytest.raises(RuntimeError):
        ob.ref_read_assignment(0, p, 3)
