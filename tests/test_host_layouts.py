"""The host layout builders (iccg_b200/csrc/host_layout.cpp), on the CPU.

Both builders split their passes over host threads, and their arrays must
not depend on the thread count.

* IC(0) layout: the arrays must equal a plain one-row-at-a-time restatement
  of the reference's extract_lower_with_diag, diag_pos and
  build_csc_from_crs (ic0.cpp:14-54, 118-151), plus the strict lower / upper
  split. L's rows and columns must also equal the oracle's IC(0) pattern.
* SELL-32 layout: the arrays must equal a one-slice-at-a-time restatement,
  including the in-unit encoding of the substitution matrices and its
  refusals.

tests/cpp/*_main.cpp run a builder on one input. They are compiled here
with g++.
"""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import iccg_b200 as ib
import iccg_b200.problems as pb
from oracle import bindings as ob

ROOT = Path(__file__).resolve().parents[1]
NAMES = ("Lp", "Li", "dpos", "Up", "Ui", "ut_src", "Sp", "Si", "s_src", "Tp", "Ti", "t_src")
ERR_DIAG = -2  # ICCG_ERR_DIAG
THREADS = (1, 2, 3, 7)


def _compile(tmp_path_factory, main: str) -> Path:
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not found")
    exe = tmp_path_factory.mktemp("layout") / main
    subprocess.run([cxx, "-O2", "-std=c++17", "-pthread", str(ROOT / f"tests/cpp/{main}.cpp"),
                    str(ROOT / "iccg_b200/csrc/host_layout.cpp"), "-o", str(exe)], check=True)
    return exe


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    return _compile(tmp_path_factory, "ic0_layout_main")


@pytest.fixture(scope="module")
def sell_driver(tmp_path_factory):
    return _compile(tmp_path_factory, "sell_layout_main")


def run_layout(exe, tmp: Path, n, rowptr, colind, val, threads):
    """(status, message) on an error, else (0, dict of arrays)."""
    src, dst = tmp / "in.bin", tmp / "out.bin"
    with open(src, "wb") as f:
        np.asarray([n, len(colind)], np.int32).tofile(f)
        np.asarray(rowptr, np.int32).tofile(f)
        np.asarray(colind, np.int32).tofile(f)
        np.asarray(val, np.float64).tofile(f)
    subprocess.run([str(exe), str(src), str(dst), str(threads)], check=True)
    raw = dst.read_bytes()
    status = int(np.frombuffer(raw[:4], np.int32)[0])
    if status:
        return status, raw[4:].decode()
    out, pos = {}, 4
    for name, dt in [(m, np.int32) for m in NAMES] + [("Lx0", np.float64)]:
        cnt = int(np.frombuffer(raw[pos:pos + 8], np.int64)[0])
        pos += 8
        size = cnt * np.dtype(dt).itemsize
        out[name] = np.frombuffer(raw[pos:pos + size], dt).copy()
        pos += size
    assert pos == len(raw)
    return 0, out


def restate(n, rowptr, colind, val):
    """The layout, one row / column at a time (small matrices only)."""
    Lp, Li, Lx0 = [0], [], []
    for i in range(n):
        for k in range(rowptr[i], rowptr[i + 1]):
            if colind[k] <= i:
                Li.append(int(colind[k]))
                Lx0.append(float(val[k]))
        Lp.append(len(Li))
    dpos = []
    for i in range(n):
        d = next((k for k in range(Lp[i], Lp[i + 1]) if Li[k] == i), -1)
        if d < 0:
            return ERR_DIAG, f"IC(0): diagonal missing at row {i}"
        dpos.append(d)
    cols = [[] for _ in range(n)]
    for i in range(n):
        for k in range(Lp[i], Lp[i + 1]):
            cols[Li[k]].append((i, k))
    Up, Ui, ut_src = [0], [], []
    for j in range(n):
        Ui += [i for i, _ in cols[j]]
        ut_src += [k for _, k in cols[j]]
        Up.append(len(Ui))
    Sp, Si, s_src = [0], [], []
    for i in range(n):
        for k in range(Lp[i], Lp[i + 1]):
            if Li[k] >= i:
                break
            Si.append(Li[k])
            s_src.append(k)
        Sp.append(len(Si))
    Tp, Ti, t_src = [0], [], []
    for j in range(n):
        for k in range(Up[j], Up[j + 1]):
            if Ui[k] > j:
                Ti.append(Ui[k])
                t_src.append(ut_src[k])
        Tp.append(len(Ti))
    arrays = dict(Lp=Lp, Li=Li, dpos=dpos, Up=Up, Ui=Ui, ut_src=ut_src, Sp=Sp, Si=Si, s_src=s_src, Tp=Tp, Ti=Ti,
                  t_src=t_src)
    out = {k: np.asarray(v, np.int32) for k, v in arrays.items()}
    out["Lx0"] = np.asarray(Lx0, np.float64)
    return 0, out


def random_pattern(n, per, seed, all_diag=True):
    """Unsorted rows, repeated columns, a repeated diagonal now and then, an
    unsymmetric pattern; with all_diag False some rows lack a diagonal."""
    rng = np.random.default_rng(seed)
    rowptr, colind = [0], []
    for i in range(n):
        row = list(rng.integers(0, n, int(rng.integers(0, per + 1))))
        if all_diag or rng.integers(0, 50):
            row.append(i)
            if rng.integers(0, 7) == 0:
                row.append(i)
        rng.shuffle(row)
        colind += row
        rowptr.append(len(colind))
    val = rng.integers(-500, 500, len(colind)) / 7.0
    return n, np.asarray(rowptr), np.asarray(colind), val


def check_all_threads(exe, tmp, n, rowptr, colind, val):
    results = [run_layout(exe, tmp, n, rowptr, colind, val, t) for t in THREADS]
    for status, out in results[1:]:
        assert status == results[0][0]
        if status:
            assert out == results[0][1]
        else:
            for k in out:
                np.testing.assert_array_equal(out[k], results[0][1][k], err_msg=k)
    return results[0]


@pytest.mark.parametrize("n,per,seed", [(0, 0, 0), (1, 0, 1), (5, 3, 2), (37, 6, 3), (300, 9, 4), (1000, 4, 5)])
def test_layout_matches_restatement_for_every_thread_count(driver, tmp_path, n, per, seed):
    n, rowptr, colind, val = random_pattern(n, per, seed)
    status, out = check_all_threads(driver, tmp_path, n, rowptr, colind, val)
    assert status == 0
    _, want = restate(n, rowptr, colind, val)
    for k in want:
        np.testing.assert_array_equal(out[k], want[k], err_msg=k)


@pytest.mark.parametrize("seed", range(6))
def test_missing_diagonal_names_first_row(driver, tmp_path, seed):
    n, rowptr, colind, val = random_pattern(400, 5, 100 + seed, all_diag=False)
    want = restate(n, rowptr, colind, val)
    assert want[0] == ERR_DIAG
    assert check_all_threads(driver, tmp_path, n, rowptr, colind, val) == want


@pytest.mark.parametrize("case", ["stencil2d", "knn_abmc", "grid3d_mc"])
def test_layout_matches_oracle_pattern(driver, tmp_path, case):
    if case == "stencil2d":
        A = ib.gen_stencil_2d5(17, 13)
    elif case == "knn_abmc":
        A = pb.make(ib.gen_knn_laplacian(600, 8, 1e-2, 3), "abmc", block_size=8).A_run
    else:
        A = pb.make(ib.gen_stencil_3d7(12, 11, 10), "piccg").A_run
    status, out = check_all_threads(driver, tmp_path, A.n, A.rowptr, A.colind, A.val)
    assert status == 0
    Lp, Li, _, Up, Ui, _ = ob.OracleIC0(A.n, A.rowptr, A.colind, A.val).export()
    for k, v in (("Lp", Lp), ("Li", Li), ("Up", Up), ("Ui", Ui)):
        np.testing.assert_array_equal(out[k], v, err_msg=k)
    _, want = restate(A.n, A.rowptr, A.colind, A.val)
    for k in want:
        np.testing.assert_array_equal(out[k], want[k], err_msg=k)


# ---------------------------------------------------------------------------
# SELL-32 layout
# ---------------------------------------------------------------------------
ERR_ARG = -1  # ICCG_ERR_ARG
SELL_NAMES = (("h_ptr", np.int32), ("h_col", np.int32), ("h_len", np.int32), ("src", np.int32),
              ("prev_only", np.uint8), ("unit_only", np.uint8))


def run_sell(exe, tmp: Path, case: dict, threads: int):
    """(1, None) when the encoding refuses the rows, (code, message) on an
    error, else (0, dict of arrays plus slots and max_nin)."""
    src, dst = tmp / "sell_in.bin", tmp / "sell_out.bin"
    parts = [[case["nq"], len(case["slices"])], np.asarray(case["slices"], np.int32).ravel(),
             [case["n"], len(case["ci"])], case["rp"], case["ci"], [case["src_map"] is not None],
             case["src_map"] if case["src_map"] is not None else [], case["q2r"], case["r2q"], case["unit_of"],
             case["step_of"], [case["encode"]]]
    with open(src, "wb") as f:
        for p in parts:
            np.asarray(p, np.int32).tofile(f)
    subprocess.run([str(exe), str(src), str(dst), str(threads)], check=True)
    raw = dst.read_bytes()
    status = int(np.frombuffer(raw[:4], np.int32)[0])
    if status == 1:
        return 1, None
    if status:
        return status, raw[4:].decode()
    out = {"slots": int(np.frombuffer(raw[4:12], np.int64)[0]), "max_nin": int(np.frombuffer(raw[12:16], np.int32)[0])}
    pos = 16
    for name, dt in SELL_NAMES:
        cnt = int(np.frombuffer(raw[pos:pos + 8], np.int64)[0])
        pos += 8
        size = cnt * np.dtype(dt).itemsize
        out[name] = np.frombuffer(raw[pos:pos + size], dt).copy()
        pos += size
    assert pos == len(raw)
    return 0, out


def restate_sell(case: dict):
    """The SELL-32 arrays, one slice and lane at a time (small inputs only)."""
    rp, ci, q2r, unit_of, step_of, enc = (case[k] for k in ("rp", "ci", "q2r", "unit_of", "step_of", "encode"))
    if enc:
        for first, cnt in case["slices"]:
            for lane in range(cnt):
                r = q2r[first + lane]
                seen_in = seen_out = False
                for k in range(rp[r], rp[r + 1]):
                    inside = unit_of[ci[k]] == unit_of[r]
                    if (enc == 1 and seen_in and not inside) or (enc == 2 and seen_out and inside):
                        return 1, None
                    seen_in |= inside
                    seen_out |= not inside
    ptr, slot = [], 0
    for first, cnt in case["slices"]:
        ptr.append(slot)
        slot += 32 * max((rp[q2r[first + l] + 1] - rp[q2r[first + l]] for l in range(cnt)), default=0)
    ptr.append(slot)
    nq = case["nq"]
    col, src, length = [0] * slot, [-1] * slot, [0] * nq
    prev_only, unit_only = ([0] * nq, [0] * nq) if enc else ([], [])
    max_nin = 0
    for s, (first, cnt) in enumerate(case["slices"]):
        for lane in range(cnt):
            q = first + lane
            r = q2r[q]
            b, L = rp[r], rp[r + 1] - rp[r]
            if L > 0xFFFF:
                return ERR_ARG, "row longer than 65535 entries"
            nin, prev = 0, True
            for j in range(L):
                pos, cj = ptr[s] + 32 * j + lane, ci[b + j]
                if enc and unit_of[cj] == unit_of[r]:
                    col[pos] = -(step_of[cj] + 1)
                    nin += 1
                    prev = prev and step_of[cj] == step_of[r] + (-1 if enc == 1 else 1)
                else:
                    col[pos] = case["r2q"][cj]
                src[pos] = case["src_map"][b + j] if case["src_map"] is not None else b + j
            length[q] = L | (nin << 16)
            max_nin = max(max_nin, nin)
            if enc:
                prev_only[q] = int(prev and nin <= 1)
                unit_only[q] = int(nin == L)
    out = {"slots": slot, "max_nin": max_nin}
    for (name, dt), v in zip(SELL_NAMES, (ptr, col, length, src, prev_only, unit_only)):
        out[name] = np.asarray(v, dt)
    return 0, out


def sell_case(n, seed, encode, use_map=False, break_order=False, long_row=0):
    """A synthetic lane-interleaved order: rows permuted into Q order, runs
    of 1-5 consecutive Q rows form a unit (step = place in the run), slices
    of 0-32 Q rows. Rows hold out-of-unit columns and same-unit columns
    (now and then exactly the previous / next step), ordered as `encode`
    needs unless break_order."""
    rng = np.random.default_rng(seed)
    q2r = rng.permutation(n)
    r2q = np.empty(n, np.int64)
    r2q[q2r] = np.arange(n)
    unit_of, step_of = np.zeros(n, np.int64), np.zeros(n, np.int64)
    members, q, u = [], 0, 0
    while q < n:
        m = min(n - q, int(rng.integers(1, 6)))
        rows = q2r[q:q + m]
        unit_of[rows] = u
        step_of[rows] = np.arange(m)
        members.append(rows)
        q, u = q + m, u + 1
    slices, q = [], 0
    while q < n:
        cnt = min(n - q, int(rng.integers(0, 33)))
        slices.append((q, cnt))
        q += cnt
    rp, ci = [0], []
    for r in range(n):
        mates = [int(x) for x in members[unit_of[r]] if x != r]
        inside = [m for m in mates if rng.integers(0, 2)]
        if mates and rng.integers(0, 3) == 0:
            want = step_of[r] + (-1 if encode == 1 else 1)
            inside = [m for m in mates if step_of[m] == want] or inside
        outside = [int(x) for x in rng.integers(0, n, int(rng.integers(0, 6))) if unit_of[x] != unit_of[r]]
        row = outside + inside if encode != 2 else inside + outside
        if break_order and inside and outside:
            row = inside + outside if encode == 1 else outside + inside
        if long_row and r == 0:
            row = [int(q2r[0])] * long_row
        ci += row
        rp.append(len(ci))
    src_map = [int(x) for x in rng.permutation(len(ci))] if use_map else None
    return {"nq": n, "slices": slices, "n": n, "rp": rp, "ci": ci, "src_map": src_map,
            "q2r": [int(x) for x in q2r], "r2q": [int(x) for x in r2q], "unit_of": [int(x) for x in unit_of],
            "step_of": [int(x) for x in step_of], "encode": encode}


def check_sell_threads(exe, tmp, case):
    results = [run_sell(exe, tmp, case, t) for t in THREADS]
    for status, out in results[1:]:
        assert status == results[0][0]
        if status == 0:
            for k in out:
                np.testing.assert_array_equal(out[k], results[0][1][k], err_msg=k)
        else:
            assert out == results[0][1]
    return results[0]


@pytest.mark.parametrize("n,seed,encode,use_map", [(1, 0, 0, False), (40, 1, 0, False), (300, 2, 0, True),
                                                   (37, 3, 1, True), (500, 4, 1, True), (500, 5, 2, True),
                                                   (64, 6, 2, False)])
def test_sell_layout_matches_restatement(sell_driver, tmp_path, n, seed, encode, use_map):
    case = sell_case(n, seed, encode, use_map)
    status, out = check_sell_threads(sell_driver, tmp_path, case)
    want_status, want = restate_sell(case)
    assert status == want_status == 0
    for k in want:
        np.testing.assert_array_equal(out[k], want[k], err_msg=k)
    if encode:
        assert out["prev_only"].any() and out["max_nin"] >= 1


@pytest.mark.parametrize("encode", [1, 2])
def test_sell_layout_refuses_rows_out_of_encoding_order(sell_driver, tmp_path, encode):
    case = sell_case(200, 10 + encode, encode, break_order=True)
    assert restate_sell(case)[0] == 1
    assert check_sell_threads(sell_driver, tmp_path, case) == (1, None)


def test_sell_layout_rejects_rows_longer_than_65535(sell_driver, tmp_path):
    case = sell_case(50, 20, 0, long_row=65536)
    want = restate_sell(case)
    assert want[0] == ERR_ARG
    assert check_sell_threads(sell_driver, tmp_path, case) == want
