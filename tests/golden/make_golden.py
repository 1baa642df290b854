"""Generate the golden fixtures in this directory from the compiled reference.

The reference (stomo0511/ICCG) ships no tests or golden vectors, so the
fixtures are outputs of the reference itself: oracle/_ref/libiccg_ref.so,
compiled from the reference sources by oracle/Makefile.  Each case runs the
reference's main() set-up for one binary variant (cg / dcg / iccg / piccg /
abmc) and records the permutation, A_run, schedule arrays, IC(0) factor, one
preconditioner application, one SpMV and a full CG solve (OpenMP with one
thread, so the long-double reductions have a fixed order).

Inputs: the reference's own 15x15 test matrix (Saad.mm, read by the
reference's reader) and small seeded stencils built by iccg_b200's
generators (their arrays are stored in the fixture, so the fixtures do not
depend on the generators staying the same).

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import bindings as ob  # noqa: E402
import iccg_b200 as ib  # noqa: E402
from iccg_b200 import problems as pb  # noqa: E402

# the reference checkout: ICCG_REFERENCE_DIR, else `reference` beside the repository
REF_DIR = Path(os.environ.get("ICCG_REFERENCE_DIR", str(ROOT.parent / "reference")))
OUT = Path(__file__).resolve().parent
VARIANT_ID = {"cg": 0, "dcg": 1, "iccg": 2, "piccg": 3, "abmc": 4}


def record(name, A: ib.CRS, variant, P=None, tol=1e-8, seed=7, b=None):
    ref = ob.ref()
    ref.ref_set_threads(1)
    v = VARIANT_ID[variant]
    if variant == "piccg":
        R = ob.RefProblem(v, A.n, A.rowptr, A.colind, A.val, P.color, P.nc)
    elif variant == "abmc":
        R = ob.RefProblem(v, A.n, A.rowptr, A.colind, A.val, P.block_of_old, P.nb, P.block_color, P.nc)
    else:
        R = ob.RefProblem(v, A.n, A.rowptr, A.colind, A.val)
    d = dict(variant=np.array(variant), n=np.array(A.n), A_rowptr=A.rowptr, A_colind=A.colind, A_val=A.val)
    rp, ci, vv = R.arun()
    d.update(run_rowptr=rp, run_colind=ci, run_val=vv)
    if variant == "piccg":
        d.update(color=P.color, nc=np.array(P.nc))
        nc, cp, rc = R.sched_mc()
        d.update(perm=R.perm(), color_ptr=cp, rows_of_color=rc)
    if variant == "abmc":
        d.update(block_of_old=P.block_of_old, block_color=P.block_color, nb=np.array(P.nb), nc=np.array(P.nc))
        nc, nb, cpb, boc, bp, rob = R.sched_abmc()
        d.update(perm=R.perm(), color_ptr_blk=cpb, blocks_of_color=boc, block_ptr=bp, rows_of_block=rob)
    if v >= 2:
        Lp, Li, Lx, Up, Ui, Ux = R.ic0()
        d.update(L_rowptr=Lp, L_colind=Li, L_val=Lx, LT_colptr=Up, LT_rowind=Ui, LT_val=Ux)
    r = ib.gen_uniform(A.n, seed)
    d.update(apply_r=r, apply_z=R.apply(r))
    xs = ib.gen_uniform(A.n, seed + 1)
    d.update(spmv_x=xs, spmv_y=R.spmv(xs))
    if b is None:
        b = np.ones(A.n)  # the reference driver's right-hand side (cg_crs.cpp:440)
    x, it, rel, cv, _ = R.cg(b, np.zeros(A.n), 10000, tol)
    d.update(cg_b=b, cg_tol=np.array(tol), cg_x=x, cg_iters=np.array(it), cg_rel=np.array(rel),
             cg_converged=np.array(cv))
    np.savez_compressed(OUT / f"{name}.npz", **d)
    print(f"{name}: n={A.n} iters={it} rel={rel:.3e}")


def main():
    if ob.ref() is None:
        raise SystemExit("compiled reference missing: run `make -C oracle` where the reference checkout exists")
    n, rp, ci, v = ob.ref_read_mm(REF_DIR / "Saad.mm")
    saad = ib.CRS.from_arrays(n, rp, ci, v)
    for var in ("cg", "dcg", "iccg"):
        record(f"saad_{var}", saad, var)
    record("saad_piccg", saad, "piccg", pb.make(saad, "piccg"))
    record("saad_abmc", saad, "abmc", pb.make(saad, "abmc", block_size=4, blocking="bfs"))
    A2 = pb.poisson2d(32)
    P2 = pb.make(A2, "piccg", seed=0)
    record("poisson2d_32_piccg", A2, "piccg", P2, b=P2.b_run)
    record("poisson2d_32_iccg", A2, "iccg", pb.make(A2, "iccg", seed=0), b=P2.b)
    A3 = pb.laplace3d_aniso(10)
    P3 = pb.make(A3, "abmc", block_size=16, blocking="bfs", seed=0)
    record("laplace3d_10_abmc16", A3, "abmc", P3, b=P3.b_run)
    P3l = pb.make(A3, "abmc", block_size=8, blocking="linear", seed=0)
    record("laplace3d_10_abmc8lin", A3, "abmc", P3l, b=P3l.b_run)
    A27 = ib.gen_diffusion27(6, 6, 6, 1e4, 3)
    P27 = pb.make(A27, "abmc", block_size=8, seed=3)
    record("diffusion27_6_abmc8", A27, "abmc", P27, b=P27.b_run)


if __name__ == "__main__":
    main()
