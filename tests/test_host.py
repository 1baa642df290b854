"""Host-side routines of iccg_b200 against the oracle (no GPU needed).

Orderings, P^T A P, expansion and schedules must equal the reference bit for
bit (the schedule arrays are the drop-in contract); readers must accept and
reject the same inputs as the reference's.
"""
import re
from pathlib import Path

import numpy as np
import pytest

import iccg_b200 as ib
import iccg_b200.problems as pb
from oracle import bindings as ob
from _util import golden_names, load_golden

ROOT = Path(__file__).resolve().parents[1]


# ---------------------------------------------------------------------------
# the C ABI library
# ---------------------------------------------------------------------------
def test_library_exports_every_declared_symbol():
    header = (ROOT / "include" / "iccg.h").read_text()
    declared = set(re.findall(r"\b(iccg_[a-z0-9_]+)\s*\(", header))
    assert len(declared) > 40
    L = ib.lib()
    missing = [s for s in sorted(declared) if not hasattr(L, s)]
    assert not missing, missing


def test_python_binds_only_declared_symbols():
    header = (ROOT / "include" / "iccg.h").read_text()
    declared = set(re.findall(r"\b(iccg_[a-z0-9_]+)\s*\(", header))
    src = (ROOT / "iccg_b200" / "__init__.py").read_text()
    bound = set(re.findall(r'"(iccg_[a-z0-9_]+)"', src))
    assert bound <= declared, bound - declared


def test_error_message_on_bad_call():
    with pytest.raises(ib.IccgError) as e:
        ib.read_matrix_market_crs("/nonexistent/file.mtx")
    assert e.value.code == ib.ERR_IO
    assert "Failed to open" in str(e.value)


# ---------------------------------------------------------------------------
# orderings vs golden fixtures and the oracle
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name", [n for n in golden_names() if "piccg" in n or "abmc" in n])
def test_setup_matches_golden(name):
    g = load_golden(name)
    A = ib.CRS.from_arrays(int(g["n"]), g["A_rowptr"], g["A_colind"], g["A_val"])
    if str(g["variant"]) == "piccg":
        P = pb.setup(A, "piccg", color=g["color"], nc=int(g["nc"]))
        assert np.array_equal(P.sched.color_ptr, g["color_ptr"])
        assert np.array_equal(P.sched.rows_of_color, g["rows_of_color"])
    else:
        P = pb.setup(A, "abmc", block_of_old=g["block_of_old"], nb=int(g["nb"]), block_color=g["block_color"],
                     nbc=int(g["nc"]))
        for k in ("color_ptr_blk", "blocks_of_color", "block_ptr", "rows_of_block"):
            assert np.array_equal(getattr(P.sched, k), g[k]), k
    assert np.array_equal(P.new_of_old, g["perm"])
    assert np.array_equal(P.A_run.rowptr, g["run_rowptr"])
    assert np.array_equal(P.A_run.colind, g["run_colind"])
    assert np.array_equal(P.A_run.val, g["run_val"])


def _random_sym(n, density, seed, zeros=False):
    rng = np.random.default_rng(seed)
    M = (rng.random((n, n)) < density) * rng.standard_normal((n, n))
    M = M + M.T
    if zeros:
        M[rng.random((n, n)) < 0.05] = 0.0
        M = np.triu(M) + np.triu(M, 1).T
    np.fill_diagonal(M, np.abs(M).sum(1) + 1.0)
    rp, ci, v = [0], [], []
    for i in range(n):
        nz = np.nonzero(M[i])[0]
        if zeros:  # keep some explicit zeros in the pattern
            extra = rng.choice(n, 2, replace=False)
            nz = np.unique(np.concatenate([nz, extra]))
        ci += list(nz)
        v += list(M[i, nz])
        rp.append(len(ci))
    return ib.CRS.from_arrays(n, rp, ci, v)


@pytest.mark.parametrize("seed", range(6))
def test_permutations_and_ptap_match_oracle(seed):
    rng = np.random.default_rng(seed)
    A = _random_sym(60 + 10 * seed, 0.08, seed, zeros=seed % 2 == 1)
    color = rng.integers(0, 5, A.n).astype(np.int32)
    p1 = ib.BuildPermutationByColor(color)
    assert np.array_equal(p1, ob.perm_by_color(color))
    nb = 9
    blk = rng.integers(0, nb, A.n).astype(np.int32)
    bcol = rng.integers(0, 3, nb).astype(np.int32)
    p2 = ib.BuildPermutationByBlockColor(blk, bcol)
    assert np.array_equal(p2, ob.perm_by_block_color(blk, bcol))
    for p in (p1, p2):
        L = ib.Permute_PtAP_LowerCRS_to_LowerCRS(A, p)
        orp, oci, ov = ob.ptap_lower(A.n, A.rowptr, A.colind, A.val, p)
        assert np.array_equal(L.rowptr, orp) and np.array_equal(L.colind, oci) and np.array_equal(L.val, ov)
        assert not np.any(L.val == 0.0)  # color.cpp:123,132 drops exact zeros
        F = ib.expand_lower_to_full(L)
        frp, fci, fv = ob.expand_lower_to_full(A.n, orp, oci, ov)
        assert np.array_equal(F.rowptr, frp) and np.array_equal(F.colind, fci) and np.array_equal(F.val, fv)
    cp, rc = ib.BuildColorPtrRows_FromPermutationAndColor(color, 5, p1)
    ocp, orc_ = ob.color_schedule(color, 5, p1)
    assert np.array_equal(cp, ocp) and np.array_equal(rc, orc_)
    s1 = ib.BuildABMCSchedule(p2, blk, bcol, nb, 3)
    s2 = ob.abmc_schedule(p2, blk, bcol, nb, 3)
    for a, b in zip(s1, s2):
        assert np.array_equal(a, b)


def _unsorted_rows(n, seed):
    """Rows in random order with repeated columns, entries on both sides of
    the diagonal and a few rows longer than 64 entries."""
    rng = np.random.default_rng(seed)
    rp, ci = [0], []
    for i in range(n):
        row = list(rng.integers(0, n, int(rng.integers(0, 6)))) + [i]
        if i % 37 == 5:
            row += list(rng.integers(0, n, 90))
        rng.shuffle(row)
        ci += row
        rp.append(len(ci))
    v = rng.integers(-3, 4, len(ci)) / 2.0  # exact sums, some of them zero
    return ib.CRS.from_arrays(n, rp, ci, v)


def _ties_in_long_rows(M):
    """True if a row of more than 16 entries repeats a column.  The
    reference sorts rows with std::sort, which keeps equal columns in input
    order only for ranges of up to 16 entries (libstdc++ sorts those by
    insertion); the oracle keeps input order always, so such rows are
    checked against the compiled reference instead."""
    for i in range(M.n):
        c = M.colind[M.rowptr[i]:M.rowptr[i + 1]]
        if len(c) > 16 and len(np.unique(c)) < len(c):
            return True
    return False


def _same(F, arrays):
    return all(np.array_equal(a, b) for a, b in zip((F.rowptr, F.colind, F.val), arrays))


@pytest.mark.parametrize("threads", ["1", "2", "3", "7"])
def test_ptap_and_expand_match_oracle_on_every_thread_count(monkeypatch, threads):
    # ICCG_HOST_THREADS forces the thread count, so small inputs take the
    # multi-threaded passes too
    monkeypatch.setenv("ICCG_HOST_THREADS", threads)
    rng = np.random.default_rng(int(threads))
    have_ref = ob.ref() is not None
    for A in (_random_sym(150, 0.05, 3, zeros=True), _unsorted_rows(400, int(threads)), pb.laplace3d_aniso(9)):
        for p in (rng.permutation(A.n).astype(np.int32), np.arange(A.n, dtype=np.int32)):
            L = ib.Permute_PtAP_LowerCRS_to_LowerCRS(A, p)
            assert _same(L, ob.ptap_lower(A.n, A.rowptr, A.colind, A.val, p))
            if have_ref:
                assert _same(L, ob.ref_ptap_lower(A.n, A.rowptr, A.colind, A.val, p))
        for M in (L, A):
            F = ib.expand_lower_to_full(M)
            if not _ties_in_long_rows(M):
                assert _same(F, ob.expand_lower_to_full(M.n, M.rowptr, M.colind, M.val))
            if have_ref:
                assert _same(F, ob.ref_expand_lower_to_full(M.n, M.rowptr, M.colind, M.val))


def _triple_row_input(n=40, row=30, reps=24, seed=0):
    """A lower CRS whose row `row` gets, after P^T A P with the identity,
    `reps` entries of one column whose sum depends on the order they are
    added in (magnitudes 1e16 and 1), among other columns: a row longer than
    16 entries with 3 or more duplicates."""
    rng = np.random.default_rng(seed)
    rp, ci, v = [0], [], []
    for i in range(n):
        cols = [i]
        vals = [4.0]
        if i == row:
            for k in range(reps):
                cols.append(3)
                vals.append([1e16, 1.0, -1e16, 1.0, 3.0, -2.0][k % 6] * (1 + k // 6))
            for c in rng.permutation(np.arange(5, row))[:12]:
                cols.append(int(c))
                vals.append(float(rng.standard_normal()))
        order = rng.permutation(len(cols))
        ci += [cols[k] for k in order]
        v += [vals[k] for k in order]
        rp.append(len(ci))
    return ib.CRS.from_arrays(n, rp, ci, v)


@pytest.mark.skipif(ob.ref() is None, reason="compiled reference not built (needs the reference checkout)")
@pytest.mark.parametrize("seed", range(4))
def test_duplicate_entries_in_long_rows_match_compiled_reference(seed, tmp_path):
    """Three or more duplicates of one entry in a row longer than 16: the
    reference sums them in the order its std::sort leaves them (color.cpp:
    111-112 per PtAP row; crs_io.cpp:27-30 over the whole COO list of the
    MatrixMarket reader).  PtAP, expand_lower_to_full and the reader must
    give the compiled reference's bits."""
    A = _triple_row_input(seed=seed)
    for p in (np.arange(A.n, dtype=np.int32), np.random.default_rng(seed).permutation(A.n).astype(np.int32)):
        L = ib.Permute_PtAP_LowerCRS_to_LowerCRS(A, p)
        assert _same(L, ob.ref_ptap_lower(A.n, A.rowptr, A.colind, A.val, p))
    F = ib.expand_lower_to_full(A)
    assert _same(F, ob.ref_expand_lower_to_full(A.n, A.rowptr, A.colind, A.val))
    # the reader: a general file listing one entry many times among others
    rng = np.random.default_rng(seed)
    lines = []
    for k in range(60):
        lines.append((7, 5, [1e16, 1.0, -1e16, 1.0, 3.0, -2.0][k % 6] * (1 + k // 6)))
    for k in range(200):
        lines.append((int(rng.integers(1, 21)), int(rng.integers(1, 21)), float(rng.standard_normal())))
    rng.shuffle(lines)
    path = tmp_path / "dups.mtx"
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"20 20 {len(lines)}\n")
        for i, j, x in lines:
            f.write(f"{i} {j} {x!r}\n")
    mine = ib.read_matrix_market_crs(str(path))
    assert _same(mine, ob.ref_read_mm(path)[1:])


def test_ptap_long_dense_row_is_not_quadratic():
    """One row of 100 000 entries in reverse column order: the per-row sort
    is O(m log m), as the reference's std::sort is."""
    import time
    n = 100_001
    rp = np.zeros(n + 1, np.int64)
    ci, v = [], []
    for i in range(n - 1):
        ci.append(i)
        v.append(4.0)
        rp[i + 1] = len(ci)
    last = n - 1
    ci += list(range(last, -1, -1))
    v += [1.0] * (last) + [4.0]
    v[-1 - last] = 4.0
    rp[n] = len(ci)
    A = ib.CRS.from_arrays(n, rp.astype(np.int32), np.array(ci, np.int32), np.array(v))
    # the long row stays the last row; its columns arrive in random order
    p = np.concatenate([np.random.default_rng(1).permutation(n - 1), [n - 1]]).astype(np.int32)
    t0 = time.perf_counter()
    L = ib.Permute_PtAP_LowerCRS_to_LowerCRS(A, p)
    dt = time.perf_counter() - t0
    assert dt < 5.0, dt
    assert L.rowptr[-1] == 2 * n - 1
    o = ob.ptap_lower(A.n, A.rowptr, A.colind, A.val, p)
    assert _same(L, o)


def test_ptap_and_expand_reject_decreasing_rowptr():
    A = ib.CRS.from_arrays(3, [0, 2, 1, 3], [0, 0, 1], [1.0, 1.0, 1.0])
    with pytest.raises(ib.IccgError) as e:
        ib.expand_lower_to_full(A)
    assert e.value.code == ib.ERR_ARG
    with pytest.raises(ib.IccgError) as e:
        ib.Permute_PtAP_LowerCRS_to_LowerCRS(A, np.array([0, 1, 2], np.int32))
    assert e.value.code == ib.ERR_ARG


def test_ptap_and_expand_reject_indices_out_of_range():
    A = ib.CRS.from_arrays(3, [0, 1, 3, 4], [0, 0, 5, 2], [1.0, 1.0, 1.0, 1.0])
    with pytest.raises(ib.IccgError) as e:
        ib.expand_lower_to_full(A)
    assert e.value.code == ib.ERR_ARG
    B = ib.CRS.from_arrays(3, [0, 1, 3, 4], [0, 0, 1, 2], [1.0, 1.0, 1.0, 1.0])
    with pytest.raises(ib.IccgError) as e:
        ib.Permute_PtAP_LowerCRS_to_LowerCRS(B, np.array([0, 3, 1], np.int32))
    assert e.value.code == ib.ERR_ARG


def test_abmc_schedule_with_empty_block():
    # a block with no rows leaves -1 at the tail of blocks_of_color (block.cpp:141)
    blk = np.array([0, 0, 2, 2, 0], np.int32)
    bcol = np.array([0, 1, 1], np.int32)
    p = ib.BuildPermutationByBlockColor(blk, bcol)
    s1 = ib.BuildABMCSchedule(p, blk, bcol, 3, 2)
    s2 = ob.abmc_schedule(p, blk, bcol, 3, 2)
    for a, b in zip(s1, s2):
        assert np.array_equal(a, b)
    assert s1[1][-1] == -1


def test_edge_cases_sizes():
    # n = 1 and a diagonal matrix
    A = ib.CRS.from_arrays(1, [0, 1], [0], [2.0])
    P = pb.setup(A, "piccg", color=[0], nc=1)
    assert P.A_run.nnz == 1
    D = ib.CRS.from_arrays(4, [0, 1, 2, 3, 4], [0, 1, 2, 3], [1.0, 2.0, 3.0, 4.0])
    c, nc = ib.color_greedy(D)
    assert nc == 1


# ---------------------------------------------------------------------------
# readers and writers
# ---------------------------------------------------------------------------
def test_matrix_market_roundtrip_and_oracle(tmp_path):
    A = pb.laplace3d_aniso(5)
    p = tmp_path / "a.mtx"
    ib.write_matrix_market(str(p), A, symmetric=True)
    B = ib.read_matrix_market_crs(str(p))
    assert np.array_equal(A.rowptr, B.rowptr) and np.array_equal(A.colind, B.colind)
    assert np.array_equal(A.val, B.val)
    n, rp, ci, v = ob.read_mm(p)
    assert np.array_equal(B.rowptr, rp) and np.array_equal(B.colind, ci) and np.array_equal(B.val, v)


def test_matrix_market_formats(tmp_path):
    p = tmp_path / "g.mtx"
    p.write_text("%%MatrixMarket matrix coordinate pattern general\n% c\n%\n3 3 4\n1 1\n\n2 2\n3 1\n3 3\n")
    A = ib.read_matrix_market_crs(str(p))
    assert A.n == 3 and list(A.colind) == [0, 1, 0, 2] and list(A.val) == [1, 1, 1, 1]
    q = tmp_path / "d.mtx"  # duplicates are summed
    q.write_text("%%MatrixMarket matrix coordinate real general\n2 2 3\n1 1 1.5\n1 1 2.5\n2 2 1\n")
    B = ib.read_matrix_market_crs(str(q))
    assert list(B.val) == [4.0, 1.0]
    n, rp, ci, v = ob.read_mm(q)
    assert list(v) == [4.0, 1.0]


def test_matrix_market_values_parse_exactly(tmp_path):
    """Entry values and indices read from MatrixMarket text are the doubles
    and integers strtod / strtoll give (correctly rounded): subnormals, the
    extremes, long mantissas, halfway cases, and the forms only strtod takes
    (a leading '+', hexadecimal, inf / nan, trailing characters after the
    number)."""
    rng = np.random.default_rng(11)
    decimal = ["0.1", "1e-310", "4.9e-324", "2.2250738585072011e-308", "1.7976931348623157e308",
               "0.1000000000000000055511151231257827021181583404541015625",
               "123456789012345678901234567890", "-0.0", "5.", ".5", "1E5", "-2.5e-3",
               "9007199254740993", "1.00000000000000011102230246251565404236316680908203125"]
    decimal += ["%.17g" % v for v in rng.standard_normal(40) * 10.0 ** rng.integers(-30, 30, 40)]
    other = {"+1.5": 1.5, "1.5abc": 1.5, "0x1p3": 8.0, "inf": float("inf"), "-INF": float("-inf")}
    toks = decimal + list(other)
    lines = "".join(f"1 {k + 1} {t}\n" for k, t in enumerate(toks))
    p = tmp_path / "v.mtx"
    p.write_text(f"%%MatrixMarket matrix coordinate real general\n1 {len(toks)} {len(toks)}\n" + lines)
    A = ib.read_matrix_market_crs(str(p))
    assert list(A.colind) == list(range(len(toks)))
    # entries are summed from 0.0 (duplicates add up, as in the reference's
    # coo_to_crs), so -0.0 reads as +0.0
    want = [float(t) + 0.0 for t in decimal] + list(other.values())
    for got, w, t in zip(A.val, want, toks):
        assert np.float64(got).tobytes() == np.float64(w).tobytes(), (t, got, w)
    # the decimal ones also as the oracle's restatement of the reference reader
    q = tmp_path / "d.mtx"
    q.write_text(f"%%MatrixMarket matrix coordinate real general\n1 {len(decimal)} {len(decimal)}\n"
                 + "".join(f"1 {k + 1} {t}\n" for k, t in enumerate(decimal)))
    B = ib.read_matrix_market_crs(str(q))
    n, rp, ci, v = ob.read_mm(q)
    assert np.array_equal(B.val.view(np.int64), np.asarray(v).view(np.int64))
    # indices: leading zeros and a sign
    r = tmp_path / "i.mtx"
    r.write_text("%%MatrixMarket matrix coordinate real general\n3 3 2\n001 +2 1.0\n+3 0003 2.0\n")
    C = ib.read_matrix_market_crs(str(r))
    assert list(C.rowptr) == [0, 1, 1, 2] and list(C.colind) == [1, 2] and list(C.val) == [1.0, 2.0]


@pytest.mark.parametrize("text,msg", [
    ("", "Empty file"),
    ("%%MatrixMarket matrix array real general\n1 1\n1\n", "coordinate"),
    ("%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1 0\n", "Unsupported field"),
    ("%%MatrixMarket matrix coordinate real hermitian\n1 1 1\n1 1 1\n", "Unsupported symmetry"),
    ("%MatrixMarket matrix coordinate real general\n1 1 1\n1 1 1\n", "Not a MatrixMarket"),
    ("%%MatrixMarket matrix coordinate real general\n\n1 1 1\n", "Invalid size line"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1\n", "Unexpected EOF"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1\n", "Index out of range"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 x 1\n", "Invalid entry line"),
])
def test_matrix_market_errors(tmp_path, text, msg):
    p = tmp_path / "bad.mtx"
    p.write_text(text)
    with pytest.raises(ib.IccgError) as e:
        ib.read_matrix_market_crs(str(p))
    assert msg in str(e.value)
    with pytest.raises(ob.OracleError):
        ob.read_mm(p)


def test_assignment_files(tmp_path):
    p = tmp_path / "x.blk"
    ib.write_assignment_1based(str(p), np.array([2, 0, 1, 1]), 3)
    v, k = ib.ReadBlockFile_1Based(str(p), 4)
    assert k == 3 and list(v) == [2, 0, 1, 1]
    w, k2 = ob.read_assignment(p, 4)
    assert np.array_equal(v, w) and k2 == 3
    bad = tmp_path / "bad.bcol"
    bad.write_text("2\n1 1\n")
    with pytest.raises(ib.IccgError):
        ib.ReadBlockColorFile_1Based(str(bad), 2)
    # duplicates overwrite (color.cpp:57-59)
    dup = tmp_path / "dup.col"
    dup.write_text("2\n1 1\n2 1\n1 2\n")
    c, nc = ib.ReadColorFile_1Based(str(dup), 2)
    assert list(c) == [1, 0] and nc == 2


# ---------------------------------------------------------------------------
# schedule validators (cg_crs.cpp:171-336)
# ---------------------------------------------------------------------------
def test_hazard_checkers_match_oracle():
    A = pb.laplace3d_aniso(6)
    P = pb.make(A, "abmc", block_size=8)
    t, byc = ib.check_interblock_same_color(A, P.block_of_old, P.block_color, P.nb, P.nc)
    assert t == 0
    h, sb, xb = ib.check_schedule_hazards(P.A_run, P.new_of_old, P.color, P.block_of_old)
    assert xb == 0 and h == sb
    # a bad block coloring: everything one color
    bad = np.zeros(P.nb, np.int32)
    t2, _ = ib.check_interblock_same_color(A, P.block_of_old, bad, P.nb, 1)
    o2 = ob.orc().orc_check_interblock_same_color(A.n, ob._ptr(A.rowptr), ob._ptr(A.colind),
                                                  ob._ptr(P.block_of_old), ob._ptr(bad), P.nb, 1, None)
    assert t2 == o2 > 0
