"""ctypes bindings of the oracle (TEST INFRASTRUCTURE ONLY).

Two CPU implementations of the ICCG hot path, used as checkers by the tests,
by ``__graft_entry__.smoke()`` and as the CPU baseline of ``bench.py``:

* ``orc``  -- oracle/_build/liboracle.so, the C restatement
  (oracle/iccg_oracle.c); rebuilt with gcc if missing;
* ``ref``  -- oracle/_ref/libiccg_ref.so, the reference's own sources
  compiled by oracle/Makefile (present only where the reference checkout was
  available at build time).

Nothing in the product package imports this module.
"""
from __future__ import annotations

import ctypes as C
import shutil
import subprocess
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
ORC_SO = HERE / "_build" / "liboracle.so"
REF_SO = HERE / "_ref" / "libiccg_ref.so"

_P, _I, _D = C.c_void_p, C.c_int, C.c_double


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class _Sched(C.Structure):
    _fields_ = [("nc", _I), ("color_ptr", _P), ("rows_of_color", _P), ("mode", _I), ("nb", _I),
                ("color_ptr_blk", _P), ("blocks_of_color", _P), ("block_ptr", _P), ("rows_of_block", _P)]


class _CGRes(C.Structure):
    _fields_ = [("iters", _I), ("rel_resid", _D), ("converged", _I)]


_orc: Optional[C.CDLL] = None
_ref: Optional[C.CDLL] = None
_ref_tried = False


def orc() -> C.CDLL:
    global _orc
    if _orc is not None:
        return _orc
    if not ORC_SO.exists():
        cc = "/usr/bin/gcc" if Path("/usr/bin/gcc").exists() else (shutil.which("gcc") or "gcc")
        ORC_SO.parent.mkdir(exist_ok=True)
        subprocess.run([cc, "-O2", "-std=c11", "-ffp-contract=off", "-fPIC", "-shared", "-o", str(ORC_SO),
                        str(HERE / "iccg_oracle.c"), "-lm"], check=True)
    L = C.CDLL(str(ORC_SO))
    sig = {
        "orc_last_error_row": (_I, []),
        "orc_perm_by_color": (_I, [_I, _P, _P]),
        "orc_perm_by_block_color": (_I, [_I, _P, _P, _P]),
        "orc_ptap_lower": (_I, [_I, _P, _P, _P, _P, _I, _P, _P, _P, C.POINTER(_I)]),
        "orc_expand_lower_to_full_nnz": (_I, [_I, _P, _P]),
        "orc_expand_lower_to_full": (_I, [_I, _P, _P, _P, _P, _P, _P]),
        "orc_color_schedule": (_I, [_I, _P, _I, _P, _P, _P]),
        "orc_abmc_schedule": (_I, [_I, _P, _P, _P, _I, _I, _P, _P, _P, _P]),
        "orc_spmv": (None, [_I, _P, _P, _P, _P, _P]),
        "orc_dot": (_D, [_I, _P, _P]),
        "orc_nrm2": (_D, [_I, _P]),
        "orc_ic0_create": (_I, [_I, _P, _P, _P, _D, C.POINTER(_P)]),
        "orc_ic0_free": (None, [_P]),
        "orc_ic0_nnz": (_I, [_P]),
        "orc_ic0_export": (None, [_P, _P, _P, _P, _P, _P, _P]),
        "orc_ic0_apply": (_I, [_P, _P, _P, C.POINTER(_Sched)]),
        "orc_jacobi_inv_diag": (None, [_I, _P, _P, _P, _P]),
        "orc_cg": (_I, [_I, _P, _P, _P, _P, _P, _I, _P, _P, C.POINTER(_Sched), _I, _D, C.POINTER(_CGRes), _P]),
        "orc_true_resid": (_D, [_I, _P, _P, _P, _P, _P]),
        "orc_check_interblock_same_color": (C.c_long, [_I, _P, _P, _P, _P, _I, _I, _P]),
        "orc_check_schedule_hazards": (C.c_long, [_I, _P, _P, _P, _P, _P, _P, _P]),
        "orc_mm_read": (_I, [C.c_char_p, C.POINTER(_P)]),
        "orc_crs_free": (None, [_P]),
        "orc_crs_n": (_I, [_P]),
        "orc_crs_nnz": (_I, [_P]),
        "orc_crs_copy": (None, [_P, _P, _P, _P]),
        "orc_read_assignment": (_I, [C.c_char_p, _I, _P, C.POINTER(_I)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _orc = L
    return L


def ref() -> Optional[C.CDLL]:
    """The compiled reference, or None where it was not built."""
    global _ref, _ref_tried
    if _ref_tried:
        return _ref
    _ref_tried = True
    if not REF_SO.exists():
        return None
    L = C.CDLL(str(REF_SO))
    sig = {
        "ref_last_error": (C.c_char_p, []),
        "ref_set_threads": (None, [_I]),
        "ref_max_threads": (_I, []),
        "ref_problem_create": (_P, [_I, _I, _P, _P, _P, _P, _I, _P, _I, _D]),
        "ref_problem_free": (None, [_P]),
        "ref_problem_n": (_I, [_P]),
        "ref_problem_nnz": (_I, [_P]),
        "ref_problem_arun": (None, [_P, _P, _P, _P]),
        "ref_problem_perm": (None, [_P, _P]),
        "ref_problem_nc": (_I, [_P]),
        "ref_problem_nb": (_I, [_P]),
        "ref_problem_sched_mc": (None, [_P, _P, _P]),
        "ref_problem_sched_abmc": (None, [_P, _P, _P, _P, _P]),
        "ref_problem_ic0_nnz": (_I, [_P]),
        "ref_problem_ic0_export": (None, [_P, _P, _P, _P, _P, _P, _P]),
        "ref_apply": (None, [_P, _P, _P]),
        "ref_spmv": (None, [_P, _P, _P]),
        "ref_dot": (_D, [_I, _P, _P]),
        "ref_nrm2": (_D, [_I, _P]),
        "ref_cg": (_I, [_P, _P, _P, _I, _D, C.POINTER(_I), C.POINTER(_D), C.POINTER(_I), C.POINTER(_D)]),
        "ref_read_mm": (_P, [C.c_char_p]),
        "ref_crs_n": (_I, [_P]),
        "ref_crs_nnz": (_I, [_P]),
        "ref_crs_copy": (None, [_P, _P, _P, _P]),
        "ref_crs_free": (None, [_P]),
        "ref_read_assignment": (_I, [_I, C.c_char_p, _I, _P, C.POINTER(_I)]),
        "ref_ptap_lower": (_P, [_I, _P, _P, _P, _P]),
        "ref_expand_lower_to_full": (_P, [_I, _P, _P, _P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _ref = L
    return L


# ---------------------------------------------------------------------------
# restatement helpers
# ---------------------------------------------------------------------------
class OracleError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


def _ck(rc):
    if rc != 0:
        raise OracleError(rc, f"oracle error {rc} (row {orc().orc_last_error_row()})")


def perm_by_color(color):
    c = _i32(color)
    out = np.zeros(len(c), np.int32)
    _ck(orc().orc_perm_by_color(len(c), _ptr(c), _ptr(out)))
    return out


def perm_by_block_color(block_of_old, block_color):
    b, c = _i32(block_of_old), _i32(block_color)
    out = np.zeros(len(b), np.int32)
    _ck(orc().orc_perm_by_block_color(len(b), _ptr(b), _ptr(c), _ptr(out)))
    return out


def ptap_lower(n, rowptr, colind, val, new_of_old):
    rp, ci, v, p = _i32(rowptr), _i32(colind), _f64(val), _i32(new_of_old)
    cap = max(len(ci), 1)
    orp = np.zeros(n + 1, np.int32)
    oci = np.zeros(cap, np.int32)
    ov = np.zeros(cap)
    nnz = C.c_int()
    _ck(orc().orc_ptap_lower(n, _ptr(rp), _ptr(ci), _ptr(v), _ptr(p), cap, _ptr(orp), _ptr(oci), _ptr(ov), C.byref(nnz)))
    return orp, oci[: nnz.value].copy(), ov[: nnz.value].copy()


def expand_lower_to_full(n, rowptr, colind, val):
    rp, ci, v = _i32(rowptr), _i32(colind), _f64(val)
    m = orc().orc_expand_lower_to_full_nnz(n, _ptr(rp), _ptr(ci))
    frp, fci, fv = np.zeros(n + 1, np.int32), np.zeros(m, np.int32), np.zeros(m)
    _ck(orc().orc_expand_lower_to_full(n, _ptr(rp), _ptr(ci), _ptr(v), _ptr(frp), _ptr(fci), _ptr(fv)))
    return frp, fci, fv


def color_schedule(color, nc, new_of_old):
    c, p = _i32(color), _i32(new_of_old)
    cp, rc = np.zeros(nc + 1, np.int32), np.zeros(len(c), np.int32)
    _ck(orc().orc_color_schedule(len(c), _ptr(c), nc, _ptr(p), _ptr(cp), _ptr(rc)))
    return cp, rc


def abmc_schedule(new_of_old, block_of_old, block_color, nb, nc):
    p, b, c = _i32(new_of_old), _i32(block_of_old), _i32(block_color)
    cpb, boc = np.zeros(nc + 1, np.int32), np.zeros(nb, np.int32)
    bp, rob = np.zeros(nb + 1, np.int32), np.zeros(len(p), np.int32)
    _ck(orc().orc_abmc_schedule(len(p), _ptr(p), _ptr(b), _ptr(c), nb, nc, _ptr(cpb), _ptr(boc), _ptr(bp), _ptr(rob)))
    return cpb, boc, bp, rob


def spmv(n, rowptr, colind, val, x):
    y = np.zeros(n)
    orc().orc_spmv(n, _ptr(_i32(rowptr)), _ptr(_i32(colind)), _ptr(_f64(val)), _ptr(_f64(x)), _ptr(y))
    return y


def dot(a, b):
    a, b = _f64(a), _f64(b)
    return orc().orc_dot(len(a), _ptr(a), _ptr(b))


def nrm2(a):
    a = _f64(a)
    return orc().orc_nrm2(len(a), _ptr(a))


def read_mm(path):
    h = C.c_void_p()
    _ck(orc().orc_mm_read(str(path).encode(), C.byref(h)))
    L = orc()
    n, nnz = L.orc_crs_n(h), L.orc_crs_nnz(h)
    rp, ci, v = np.zeros(n + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz)
    L.orc_crs_copy(h, _ptr(rp), _ptr(ci), _ptr(v))
    L.orc_crs_free(h)
    return n, rp, ci, v


def read_assignment(path, n_expected):
    out = np.zeros(n_expected, np.int32)
    k = C.c_int()
    _ck(orc().orc_read_assignment(str(path).encode(), n_expected, _ptr(out), C.byref(k)))
    return out, k.value


class OracleIC0:
    """IC0 of the restatement: factor plus apply (ic0.cpp)."""

    def __init__(self, n, rowptr, colind, val, shift=0.0):
        self.n = n
        self._keep = (_i32(rowptr), _i32(colind), _f64(val))
        h = C.c_void_p()
        _ck(orc().orc_ic0_create(n, _ptr(self._keep[0]), _ptr(self._keep[1]), _ptr(self._keep[2]), shift, C.byref(h)))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            orc().orc_ic0_free(self.h)
            self.h = None

    def export(self):
        m = orc().orc_ic0_nnz(self.h)
        Lp, Up = np.zeros(self.n + 1, np.int32), np.zeros(self.n + 1, np.int32)
        Li, Ui, Lx, Ux = np.zeros(m, np.int32), np.zeros(m, np.int32), np.zeros(m), np.zeros(m)
        orc().orc_ic0_export(self.h, _ptr(Lp), _ptr(Li), _ptr(Lx), _ptr(Up), _ptr(Ui), _ptr(Ux))
        return Lp, Li, Lx, Up, Ui, Ux

    def apply(self, r, sched=None):
        r = _f64(r)
        z = np.zeros(self.n)
        s, keep = make_sched(sched)
        _ck(orc().orc_ic0_apply(self.h, _ptr(r), _ptr(z), C.byref(s) if s is not None else None))
        del keep
        return z


def make_sched(sched):
    """A ColorSchedule-like object (attributes nc, color_ptr, ...) -> C struct."""
    if sched is None:
        return None, None
    keep = []

    def p(a):
        if a is None:
            return None
        a = _i32(a)
        keep.append(a)
        return _ptr(a)

    s = _Sched(int(sched.nc), p(sched.color_ptr), p(sched.rows_of_color), int(sched.mode), int(sched.nb),
               p(sched.color_ptr_blk), p(sched.blocks_of_color), p(sched.block_ptr), p(sched.rows_of_block))
    return s, keep


def cg(n, rowptr, colind, val, b, x0, kind, max_iter, tol, ic0: Optional[OracleIC0] = None, sched=None,
       history=False):
    """conjugate_gradient of the restatement; kind 0 Identity, 1 Jacobi, 2 IC0.
    Returns (x, iters, rel_resid, converged, history-or-None)."""
    rp, ci, v = _i32(rowptr), _i32(colind), _f64(val)
    b = _f64(b)
    x = _f64(x0).copy()
    inv = None
    if kind == 1:
        inv = np.zeros(n)
        orc().orc_jacobi_inv_diag(n, _ptr(rp), _ptr(ci), _ptr(v), _ptr(inv))
    s, keep = make_sched(sched)
    res = _CGRes()
    hist = np.zeros(max_iter + 1) if history else None
    _ck(orc().orc_cg(n, _ptr(rp), _ptr(ci), _ptr(v), _ptr(b), _ptr(x), kind, _ptr(inv),
                     ic0.h if ic0 is not None else None, C.byref(s) if s is not None else None,
                     max_iter, tol, C.byref(res), _ptr(hist)))
    del keep
    if hist is not None:
        hist = hist[: res.iters + 1]
    return x, res.iters, res.rel_resid, bool(res.converged), hist


def true_resid(n, rowptr, colind, val, x, b):
    return orc().orc_true_resid(n, _ptr(_i32(rowptr)), _ptr(_i32(colind)), _ptr(_f64(val)), _ptr(_f64(x)), _ptr(_f64(b)))


# ---------------------------------------------------------------------------
# the compiled reference
# ---------------------------------------------------------------------------
class RefProblem:
    """The reference's main() set-up (cg_crs.cpp:377-484) for one variant:
    0 cg, 1 dcg, 2 iccg, 3 piccg (MC), 4 abmc."""

    def __init__(self, variant, n, rowptr, colind, val, color0=None, k0=0, bcolor0=None, nc=0, shift=0.0):
        L = ref()
        if L is None:
            raise RuntimeError("compiled reference not available")
        self._keep = [_i32(rowptr), _i32(colind), _f64(val)]
        c0 = None if color0 is None else _i32(color0)
        bc = None if bcolor0 is None else _i32(bcolor0)
        self._keep += [c0, bc]
        h = L.ref_problem_create(variant, n, _ptr(self._keep[0]), _ptr(self._keep[1]), _ptr(self._keep[2]),
                                 _ptr(c0), int(k0), _ptr(bc), int(nc), float(shift))
        if not h:
            raise RuntimeError("reference: " + L.ref_last_error().decode())
        self.h = h
        self.variant = variant
        self.n = L.ref_problem_n(h)

    def __del__(self):
        if getattr(self, "h", None):
            ref().ref_problem_free(self.h)
            self.h = None

    def arun(self):
        L = ref()
        nnz = L.ref_problem_nnz(self.h)
        rp, ci, v = np.zeros(self.n + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz)
        L.ref_problem_arun(self.h, _ptr(rp), _ptr(ci), _ptr(v))
        return rp, ci, v

    def perm(self):
        p = np.zeros(self.n, np.int32)
        ref().ref_problem_perm(self.h, _ptr(p))
        return p

    def sched_mc(self):
        L = ref()
        nc = L.ref_problem_nc(self.h)
        cp, rc = np.zeros(nc + 1, np.int32), np.zeros(self.n, np.int32)
        L.ref_problem_sched_mc(self.h, _ptr(cp), _ptr(rc))
        return nc, cp, rc

    def sched_abmc(self):
        L = ref()
        nc, nb = L.ref_problem_nc(self.h), L.ref_problem_nb(self.h)
        cpb, boc = np.zeros(nc + 1, np.int32), np.zeros(nb, np.int32)
        bp, rob = np.zeros(nb + 1, np.int32), np.zeros(self.n, np.int32)
        L.ref_problem_sched_abmc(self.h, _ptr(cpb), _ptr(boc), _ptr(bp), _ptr(rob))
        return nc, nb, cpb, boc, bp, rob

    def ic0(self):
        L = ref()
        m = L.ref_problem_ic0_nnz(self.h)
        Lp, Up = np.zeros(self.n + 1, np.int32), np.zeros(self.n + 1, np.int32)
        Li, Ui, Lx, Ux = np.zeros(m, np.int32), np.zeros(m, np.int32), np.zeros(m), np.zeros(m)
        L.ref_problem_ic0_export(self.h, _ptr(Lp), _ptr(Li), _ptr(Lx), _ptr(Up), _ptr(Ui), _ptr(Ux))
        return Lp, Li, Lx, Up, Ui, Ux

    def apply(self, r):
        r = _f64(r)
        z = np.zeros(self.n)
        ref().ref_apply(self.h, _ptr(r), _ptr(z))
        return z

    def spmv(self, x):
        x = _f64(x)
        y = np.zeros(self.n)
        ref().ref_spmv(self.h, _ptr(x), _ptr(y))
        return y

    def cg(self, b, x0, max_iter, tol):
        b = _f64(b)
        x = _f64(x0).copy()
        it, rel, cv, us = C.c_int(), C.c_double(), C.c_int(), C.c_double()
        ref().ref_cg(self.h, _ptr(b), _ptr(x), int(max_iter), float(tol), C.byref(it), C.byref(rel), C.byref(cv),
                     C.byref(us))
        return x, it.value, rel.value, bool(cv.value), us.value


def ref_read_mm(path):
    L = ref()
    h = L.ref_read_mm(str(path).encode())
    if not h:
        raise RuntimeError(L.ref_last_error().decode())
    n, nnz = L.ref_crs_n(h), L.ref_crs_nnz(h)
    rp, ci, v = np.zeros(n + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz)
    L.ref_crs_copy(h, _ptr(rp), _ptr(ci), _ptr(v))
    L.ref_crs_free(h)
    return n, rp, ci, v


def _ref_crs_take(h):
    L = ref()
    if not h:
        raise RuntimeError(L.ref_last_error().decode())
    n, nnz = L.ref_crs_n(h), L.ref_crs_nnz(h)
    rp, ci, v = np.zeros(n + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz)
    L.ref_crs_copy(h, _ptr(rp), _ptr(ci), _ptr(v))
    L.ref_crs_free(h)
    return rp, ci, v


def ref_ptap_lower(n, rowptr, colind, val, new_of_old):
    """The reference's Permute_PtAP_LowerCRS_to_LowerCRS (color.cpp:66-141)."""
    rp, ci, v, p = _i32(rowptr), _i32(colind), _f64(val), _i32(new_of_old)
    return _ref_crs_take(ref().ref_ptap_lower(n, _ptr(rp), _ptr(ci), _ptr(v), _ptr(p)))


def ref_expand_lower_to_full(n, rowptr, colind, val):
    """The reference's expand_lower_to_full (crs_io.cpp:163-227)."""
    rp, ci, v = _i32(rowptr), _i32(colind), _f64(val)
    return _ref_crs_take(ref().ref_expand_lower_to_full(n, _ptr(rp), _ptr(ci), _ptr(v)))


def ref_read_assignment(kind, path, n_expected):
    out = np.zeros(n_expected, np.int32)
    k = C.c_int()
    rc = ref().ref_read_assignment(kind, str(path).encode(), n_expected, _ptr(out), C.byref(k))
    if rc != 0:
        raise RuntimeError(ref().ref_last_error().decode())
    return out, k.value
