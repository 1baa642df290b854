"""iccg_b200 -- preconditioned CG on CRS matrices for NVIDIA B200 (sm_100a).

Python mirror of the interface of stomo0511/ICCG, over the C ABI of
``include/iccg.h`` (``iccg_b200/_lib/libiccg_b200.so``):

* ``CRS`` and ``read_matrix_market_crs`` / ``expand_lower_to_full``
  (crs_io.hpp:10-56)
* the color and block readers, permutations, ``Permute_PtAP_...`` and the
  schedule builders (color.hpp, block.hpp), bit-exact with the reference
* ``ColorSchedule`` (color.hpp:9-22)
* ``Identity``, ``Jacobi``, ``IC0`` with ``apply(r, z, sched)`` and ``name()``
  (precond.hpp, ic0.hpp), computed on the GPU
* ``conjugate_gradient(A, b, x, M, max_iter, tol, sched)`` returning
  ``CGResult`` (cg_crs.cpp:82-162), run on the GPU

The compute path is the CUDA library only; importing a GPU entry point
without the built library raises ``ImportError`` instead of falling back.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from pathlib import Path
from typing import List, Optional, Sequence

import numpy as np

__all__ = [
    "CRS", "ColorSchedule", "CGResult", "IccgError", "lib",
    "read_matrix_market_crs", "write_matrix_market", "expand_lower_to_full",
    "ReadColorFile_1Based", "ReadBlockFile_1Based", "ReadBlockColorFile_1Based",
    "write_assignment_1based",
    "BuildPermutationByColor", "BuildPermutationByBlockColor",
    "Permute_PtAP_LowerCRS_to_LowerCRS", "Permute_PtAP_full_gpu", "BuildColorPtrRows_FromPermutationAndColor",
    "BuildABMCSchedule", "check_interblock_same_color", "check_schedule_hazards",
    "gen_stencil_2d5", "gen_stencil_3d7", "gen_diffusion27", "gen_knn_laplacian", "gen_uniform",
    "color_greedy", "block_partition", "color_blocks", "host_spmv",
    "Context", "Identity", "Jacobi", "IC0", "conjugate_gradient",
    "PRECOND_NONE", "PRECOND_JACOBI", "PRECOND_IC0", "STORE_FP64", "STORE_FP32",
    "MODE_PLAIN", "MODE_FUSED", "Batch",
]

_LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libiccg_b200.so"

OK = 0
ERR_ARG, ERR_DIAG, ERR_PIVOT_ZERO, ERR_PIVOT_NONPOS = -1, -2, -3, -4
ERR_IO, ERR_NOMEM, ERR_CUDA, ERR_STATE, ERR_SCHEDULE, ERR_NONFINITE = -5, -6, -7, -8, -9, -10
PRECOND_NONE, PRECOND_JACOBI, PRECOND_IC0 = 0, 1, 2
STORE_FP64, STORE_FP32 = 0, 1
MODE_PLAIN, MODE_FUSED = 0, 1
OPT_TILED = 0
OPT_SWEEP = 1
OPT_PDL = 2
OPT_STAGE_KB = 3
OPT_STAGE_BUFS = 4
OPT_PERSIST = 5
OPT_FUSE_UPDATE = 6
OPT_DEFER_X = 7
OPT_SPMV_PACK = 8
OPT_STAGE_ROWS = 9
OPT_SPMV_TPR = 10
OPT_EARLY = 11
OPT_UPDATE_CHAIN = 12
STATUS_NAMES = {0: "converged", 1: "breakdown", 2: "max_iter", 3: "nonfinite"}


class IccgError(RuntimeError):
    """A failing status of the C ABI (the reference throws std::runtime_error)."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


class _Result(C.Structure):
    _fields_ = [
        ("iters", C.c_int), ("converged", C.c_int), ("status", C.c_int), ("n_replacements", C.c_int),
        ("rel_resid", C.c_double), ("true_rel_resid", C.c_double), ("solve_ms", C.c_double),
    ]


class _Opts(C.Structure):
    _fields_ = [("mode", C.c_int), ("storage", C.c_int), ("rr_interval", C.c_int), ("graph_iters", C.c_int)]


_lib: Optional[C.CDLL] = None
_P = C.c_void_p
_I = C.c_int
_D = C.c_double


def lib() -> C.CDLL:
    """The loaded C ABI library (raises ImportError when it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        raise ImportError(f"iccg_b200 CUDA library not built: {_LIB_PATH} (run `python -m iccg_b200.build`)")
    L = C.CDLL(str(_LIB_PATH))
    sig = {
        "iccg_last_error": (C.c_char_p, []),
        "iccg_mm_read": (_I, [C.c_char_p, C.POINTER(_P)]),
        "iccg_mm_write": (_I, [C.c_char_p, _I, _P, _P, _P, _I]),
        "iccg_crs_create": (_I, [_I, _P, _P, _P, C.POINTER(_P)]),
        "iccg_crs_dims": (_I, [_P, C.POINTER(_I), C.POINTER(_I)]),
        "iccg_crs_copy": (_I, [_P, _P, _P, _P]),
        "iccg_crs_free": (None, [_P]),
        "iccg_read_assignment": (_I, [_I, C.c_char_p, _I, _P, C.POINTER(_I)]),
        "iccg_write_assignment": (_I, [C.c_char_p, _I, _P, _I]),
        "iccg_perm_by_color": (_I, [_I, _P, _P]),
        "iccg_perm_by_block_color": (_I, [_I, _I, _P, _P, _P]),
        "iccg_ptap_lower": (_I, [_I, _P, _P, _P, _P, _I, _P, _P, _P, C.POINTER(_I)]),
        "iccg_expand_lower_nnz": (_I, [_I, _P, _P, C.POINTER(_I)]),
        "iccg_expand_lower_to_full": (_I, [_I, _P, _P, _P, _P, _P, _P]),
        "iccg_ptap_full_gpu": (_I, [_I, _I, _P, _P, _P, _P, _I, _P, _P, _P, C.POINTER(_I), C.POINTER(_I)]),
        "iccg_color_schedule": (_I, [_I, _P, _I, _P, _P, _P]),
        "iccg_abmc_schedule": (_I, [_I, _P, _P, _P, _I, _I, _P, _P, _P, _P]),
        "iccg_check_interblock_same_color": (C.c_longlong, [_I, _P, _P, _P, _P, _I, _I, _P]),
        "iccg_check_schedule_hazards": (C.c_longlong, [_I, _P, _P, _P, _P, _P, _P, _P]),
        "iccg_gen_stencil": (_I, [_I, _I, _I, _I, _D, _D, _D, C.POINTER(_P)]),
        "iccg_gen_diffusion27": (_I, [_I, _I, _I, _D, C.c_ulonglong, C.POINTER(_P)]),
        "iccg_gen_knn_laplacian": (_I, [_I, _I, _D, C.c_ulonglong, C.POINTER(_P)]),
        "iccg_gen_uniform": (_I, [_I, C.c_ulonglong, _P]),
        "iccg_host_spmv": (_I, [_I, _P, _P, _P, _P, _P]),
        "iccg_color_greedy": (_I, [_I, _P, _P, _P, C.POINTER(_I)]),
        "iccg_block_partition": (_I, [_I, _P, _P, _I, _I, _P, C.POINTER(_I)]),
        "iccg_color_blocks": (_I, [_I, _P, _P, _P, _I, _P, C.POINTER(_I)]),
        "iccg_ctx_create": (_I, [_I, C.POINTER(_P)]),
        "iccg_ctx_destroy": (_I, [_P]),
        "iccg_ctx_last_error": (C.c_char_p, [_P]),
        "iccg_ctx_stream": (_P, [_P]),
        "iccg_ctx_launch_count": (C.c_longlong, [_P]),
        "iccg_ctx_device_bytes": (C.c_longlong, [_P]),
        "iccg_ctx_set_option": (_I, [_P, _I, C.c_longlong]),
        "iccg_matrix_upload": (_I, [_P, _I, _P, _P, _P]),
        "iccg_schedule_mc": (_I, [_P, _I, _P, _P]),
        "iccg_schedule_abmc": (_I, [_P, _I, _I, _P, _P, _P, _P]),
        "iccg_schedule_none": (_I, [_P]),
        "iccg_precond_build": (_I, [_P, _I, _D, _I]),
        "iccg_precond_shift": (_D, [_P]),
        "iccg_precond_apply": (_I, [_P, _P, _P, _I]),
        "iccg_precond_apply_dev": (_I, [_P, _P, _P, _I]),
        "iccg_precond_nnz": (_I, [_P, C.POINTER(_I)]),
        "iccg_precond_export": (_I, [_P, _P, _P, _P, _P, _P, _P]),
        "iccg_spmv": (_I, [_P, _P, _P, _I]),
        "iccg_spmv_dev": (_I, [_P, _P, _P, _I]),
        "iccg_dot_dev": (_I, [_P, _I, _P, _P, C.POINTER(_D)]),
        "iccg_dot_dev_noalloc": (_I, [_I, _P, _P, _P, _P]),
        "iccg_solve": (_I, [_P, _P, _P, _I, _D, C.POINTER(_Opts), C.POINTER(_Result)]),
        "iccg_solve_dev": (_I, [_P, _P, _P, _I, _D, C.POINTER(_Opts), C.POINTER(_Result)]),
        "iccg_profile_enable": (_I, [_P, _I]),
        "iccg_profile_read": (_I, [_P, _I, C.POINTER(_D), C.POINTER(C.c_longlong)]),
        "iccg_sweep_plan": (_I, [_P, _I, _I, _P, _P, _I, C.POINTER(_I)]),
        "iccg_batch_create": (_I, [_I, C.POINTER(_P)]),
        "iccg_batch_destroy": (_I, [_P]),
        "iccg_batch_last_error": (C.c_char_p, [_P]),
        "iccg_batch_launch_count": (C.c_longlong, [_P]),
        "iccg_batch_device_bytes": (C.c_longlong, [_P]),
        "iccg_batch_device_ms": (_D, [_P]),
        "iccg_batch_add_system": (_I, [_P, _P, C.POINTER(_I)]),
        "iccg_batch_clear": (_I, [_P]),
        "iccg_batch_solve": (_I, [_P, _I, _P, _P, _P, _I, _D, C.POINTER(_Opts), _P]),
        "iccg_batch_remove_system": (_I, [_P, _I]),
        "iccg_batch_open": (_I, [_P, _I, C.POINTER(_Opts)]),
        "iccg_batch_submit": (_I, [_P, _I, _P, _P, _I, _D, C.POINTER(_I)]),
        "iccg_batch_step": (_I, [_P, _P, _I, C.POINTER(_I), C.POINTER(_I)]),
        "iccg_batch_retire": (_I, [_P, _I, _P, _P, _P]),
        "iccg_device_memory": (_I, [_I, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def exported_symbols() -> list[str]:
    """Every C ABI function this module binds (used by the ABI tests)."""
    lib()
    return [n for n in dir(_lib) if n.startswith("iccg_")]


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _check(rc: int, ctx=None):
    if rc != OK:
        if ctx is not None:
            msg = lib().iccg_ctx_last_error(ctx).decode(errors="replace")
        else:
            msg = lib().iccg_last_error().decode(errors="replace")
        raise IccgError(rc, msg)


# ---------------------------------------------------------------------------
# CRS (crs_io.hpp:10-49)
# ---------------------------------------------------------------------------
@dataclass
class CRS:
    n: int
    rowptr: np.ndarray
    colind: np.ndarray
    val: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.rowptr[self.n])

    @staticmethod
    def from_arrays(n, rowptr, colind, val) -> "CRS":
        return CRS(int(n), _i32(rowptr), _i32(colind), _f64(val))

    def to_dense(self) -> np.ndarray:
        A = np.zeros((self.n, self.n))
        for i in range(self.n):
            for k in range(self.rowptr[i], self.rowptr[i + 1]):
                A[i, self.colind[k]] += self.val[k]
        return A


def _take_crs(h: C.c_void_p) -> CRS:
    L = lib()
    n, nnz = C.c_int(), C.c_int()
    L.iccg_crs_dims(h, C.byref(n), C.byref(nnz))
    rp = np.zeros(n.value + 1, np.int32)
    ci = np.zeros(nnz.value, np.int32)
    v = np.zeros(nnz.value, np.float64)
    L.iccg_crs_copy(h, _ptr(rp), _ptr(ci), _ptr(v))
    L.iccg_crs_free(h)
    return CRS(n.value, rp, ci, v)


def read_matrix_market_crs(path: str) -> CRS:
    """read_matrix_market_crs (crs_io.hpp:52, crs_io.cpp:73-159)."""
    h = C.c_void_p()
    _check(lib().iccg_mm_read(os.fsencode(path), C.byref(h)))
    return _take_crs(h)


def write_matrix_market(path: str, A: CRS, symmetric: bool = True) -> None:
    _check(lib().iccg_mm_write(os.fsencode(path), A.n, _ptr(A.rowptr), _ptr(A.colind), _ptr(A.val), int(symmetric)))


def expand_lower_to_full(L_: CRS) -> CRS:
    """expand_lower_to_full (crs_io.hpp:56, crs_io.cpp:163-227)."""
    L = lib()
    nnz = C.c_int()
    _check(L.iccg_expand_lower_nnz(L_.n, _ptr(L_.rowptr), _ptr(L_.colind), C.byref(nnz)))
    rp = np.zeros(L_.n + 1, np.int32)
    ci = np.zeros(nnz.value, np.int32)
    v = np.zeros(nnz.value, np.float64)
    _check(L.iccg_expand_lower_to_full(L_.n, _ptr(L_.rowptr), _ptr(L_.colind), _ptr(L_.val), _ptr(rp), _ptr(ci), _ptr(v)))
    return CRS(L_.n, rp, ci, v)


# ---------------------------------------------------------------------------
# readers (color.cpp:14-47, block.cpp:15-89)
# ---------------------------------------------------------------------------
def _read_assign(kind: int, path: str, n_expected: int):
    out = np.zeros(n_expected, np.int32)
    k = C.c_int()
    _check(lib().iccg_read_assignment(kind, os.fsencode(path), n_expected, _ptr(out), C.byref(k)))
    return out, k.value


def ReadColorFile_1Based(path: str, n_expected: int):
    """Returns (color[0-based], nc)."""
    return _read_assign(0, path, n_expected)


def ReadBlockFile_1Based(path: str, n_expected: int):
    """Returns (block_of_old[0-based], nb)."""
    return _read_assign(1, path, n_expected)


def ReadBlockColorFile_1Based(path: str, nb_expected: int):
    """Returns (block_color[0-based], nc)."""
    return _read_assign(2, path, nb_expected)


def write_assignment_1based(path: str, values0, k: int) -> None:
    v = _i32(values0)
    _check(lib().iccg_write_assignment(os.fsencode(path), len(v), _ptr(v), int(k)))


# ---------------------------------------------------------------------------
# orderings and schedules (color.cpp, block.cpp)
# ---------------------------------------------------------------------------
def BuildPermutationByColor(color) -> np.ndarray:
    c = _i32(color)
    out = np.zeros(len(c), np.int32)
    _check(lib().iccg_perm_by_color(len(c), _ptr(c), _ptr(out)))
    return out


def BuildPermutationByBlockColor(block_of_old, block_color) -> np.ndarray:
    b, c = _i32(block_of_old), _i32(block_color)
    out = np.zeros(len(b), np.int32)
    _check(lib().iccg_perm_by_block_color(len(b), len(c), _ptr(b), _ptr(c), _ptr(out)))
    return out


def Permute_PtAP_LowerCRS_to_LowerCRS(A: CRS, new_of_old) -> CRS:
    p = _i32(new_of_old)
    cap = max(int(A.nnz), 1)
    rp = np.zeros(A.n + 1, np.int32)
    ci = np.zeros(cap, np.int32)
    v = np.zeros(cap, np.float64)
    nnz = C.c_int()
    _check(lib().iccg_ptap_lower(A.n, _ptr(A.rowptr), _ptr(A.colind), _ptr(A.val), _ptr(p), cap,
                                 _ptr(rp), _ptr(ci), _ptr(v), C.byref(nnz)))
    # views of the leading entries: the result is short-lived (expanded to
    # the full matrix next), so the unused tail is kept rather than copied
    return CRS(A.n, rp, ci[: nnz.value], v[: nnz.value])


def Permute_PtAP_full_gpu(A: CRS, new_of_old, device: int = 0):
    """expand_lower_to_full(Permute_PtAP_LowerCRS_to_LowerCRS(A, new_of_old))
    computed on the GPU (iccg_ptap_full_gpu): the caller's A_run, the same
    bits as the host routines.  Returns (CRS, computed_on_device)."""
    p = _i32(new_of_old)
    cap = max(2 * int(A.nnz), 1)
    rp = np.zeros(A.n + 1, np.int32)
    ci = np.zeros(cap, np.int32)
    v = np.zeros(cap, np.float64)
    nnz, dev = C.c_int(), C.c_int()
    _check(lib().iccg_ptap_full_gpu(int(device), A.n, _ptr(A.rowptr), _ptr(A.colind), _ptr(A.val), _ptr(p), cap,
                                    _ptr(rp), _ptr(ci), _ptr(v), C.byref(nnz), C.byref(dev)))
    return CRS(A.n, rp, ci[: nnz.value].copy(), v[: nnz.value].copy()), bool(dev.value)


def BuildColorPtrRows_FromPermutationAndColor(color, nc: int, new_of_old):
    c, p = _i32(color), _i32(new_of_old)
    cp = np.zeros(nc + 1, np.int32)
    rc = np.zeros(len(c), np.int32)
    _check(lib().iccg_color_schedule(len(c), _ptr(c), int(nc), _ptr(p), _ptr(cp), _ptr(rc)))
    return cp, rc


def BuildABMCSchedule(new_of_old, block_of_old, block_color, nb: int, nc: int):
    p, b, c = _i32(new_of_old), _i32(block_of_old), _i32(block_color)
    cpb = np.zeros(nc + 1, np.int32)
    boc = np.zeros(nb, np.int32)
    bp = np.zeros(nb + 1, np.int32)
    rob = np.zeros(len(p), np.int32)
    _check(lib().iccg_abmc_schedule(len(p), _ptr(p), _ptr(b), _ptr(c), int(nb), int(nc),
                                    _ptr(cpb), _ptr(boc), _ptr(bp), _ptr(rob)))
    return cpb, boc, bp, rob


def check_interblock_same_color(A: CRS, block_of_old, block_color, nb: int, nc: int):
    """DebugCheck_InterBlockSameColorEdges (cg_crs.cpp:171-224): (total, per-color)."""
    b, c = _i32(block_of_old), _i32(block_color)
    byc = np.zeros(nc, np.int64)
    t = lib().iccg_check_interblock_same_color(A.n, _ptr(A.rowptr), _ptr(A.colind), _ptr(b), _ptr(c), nb, nc, _ptr(byc))
    if t < 0:
        raise IccgError(int(t), "id out of range")
    return int(t), byc


def check_schedule_hazards(Ap_full: CRS, new_of_old, color_old, block_of_old=None):
    """DebugCheck_ScheduleHazards_OnLower (cg_crs.cpp:259-336): (total, same_block, cross_block)."""
    p, c = _i32(new_of_old), _i32(color_old)
    b = None if block_of_old is None else _i32(block_of_old)
    sb, xb = C.c_longlong(), C.c_longlong()
    t = lib().iccg_check_schedule_hazards(Ap_full.n, _ptr(Ap_full.rowptr), _ptr(Ap_full.colind), _ptr(p), _ptr(c),
                                          _ptr(b), C.byref(sb), C.byref(xb))
    if t < 0:
        raise IccgError(int(t), "new_of_old out of range")
    return int(t), sb.value, xb.value


# ---------------------------------------------------------------------------
# generators
# ---------------------------------------------------------------------------
def _gen(fn, *args) -> CRS:
    h = C.c_void_p()
    _check(fn(*args, C.byref(h)))
    return _take_crs(h)


def gen_stencil_2d5(nx: int, ny: int, wx: float = 1.0, wy: float = 1.0) -> CRS:
    return _gen(lib().iccg_gen_stencil, 0, nx, ny, 1, wx, wy, 0.0)


def gen_stencil_3d7(nx: int, ny: int, nz: int, wx: float = 1.0, wy: float = 1.0, wz: float = 1.0) -> CRS:
    return _gen(lib().iccg_gen_stencil, 1, nx, ny, nz, wx, wy, wz)


def gen_diffusion27(nx: int, ny: int, nz: int, contrast: float = 1e4, seed: int = 0) -> CRS:
    return _gen(lib().iccg_gen_diffusion27, nx, ny, nz, contrast, seed)


def gen_knn_laplacian(npts: int, k: int = 8, diag_shift: float = 1e-2, seed: int = 0) -> CRS:
    return _gen(lib().iccg_gen_knn_laplacian, npts, k, diag_shift, seed)


def gen_uniform(n: int, seed: int) -> np.ndarray:
    out = np.zeros(n, np.float64)
    _check(lib().iccg_gen_uniform(n, seed, _ptr(out)))
    return out


def host_spmv(A: CRS, x) -> np.ndarray:
    """y = A x on the host with spmv's rounding (cg_crs.cpp:68-77)."""
    x = _f64(x)
    y = np.zeros(A.n)
    _check(lib().iccg_host_spmv(A.n, _ptr(A.rowptr), _ptr(A.colind), _ptr(A.val), _ptr(x), _ptr(y)))
    return y


def color_greedy(A: CRS):
    color = np.zeros(A.n, np.int32)
    nc = C.c_int()
    _check(lib().iccg_color_greedy(A.n, _ptr(A.rowptr), _ptr(A.colind), _ptr(color), C.byref(nc)))
    return color, nc.value


def block_partition(A: CRS, block_size: int, method: str = "bfs"):
    m = {"linear": 0, "bfs": 1}[method]
    b = np.zeros(A.n, np.int32)
    nb = C.c_int()
    _check(lib().iccg_block_partition(A.n, _ptr(A.rowptr), _ptr(A.colind), block_size, m, _ptr(b), C.byref(nb)))
    return b, nb.value


def color_blocks(A: CRS, block_of_old, nb: int):
    b = _i32(block_of_old)
    c = np.zeros(nb, np.int32)
    nc = C.c_int()
    _check(lib().iccg_color_blocks(A.n, _ptr(A.rowptr), _ptr(A.colind), _ptr(b), nb, _ptr(c), C.byref(nc)))
    return c, nc.value


# ---------------------------------------------------------------------------
# ColorSchedule (color.hpp:9-22)
# ---------------------------------------------------------------------------
@dataclass
class ColorSchedule:
    MC_NODE = 0
    ABMC_BLOCK = 1
    nc: int = 0
    color_ptr: Optional[np.ndarray] = None
    rows_of_color: Optional[np.ndarray] = None
    mode: int = 0
    nb: int = 0
    color_ptr_blk: Optional[np.ndarray] = None
    blocks_of_color: Optional[np.ndarray] = None
    block_ptr: Optional[np.ndarray] = None
    rows_of_block: Optional[np.ndarray] = None

    def kind(self) -> int:
        """Dispatch of IC0::apply (ic0.cpp:366-393): 0 none, 1 MC, 2 ABMC."""
        if self.nc <= 0:
            return 0
        if (self.mode == self.ABMC_BLOCK and self.color_ptr_blk is not None and self.blocks_of_color is not None
                and self.block_ptr is not None and self.rows_of_block is not None):
            return 2
        if self.color_ptr is not None and self.rows_of_color is not None:
            return 1
        return 0


@dataclass
class CGResult:
    """CGResult (cg_crs.cpp:82-86) plus the device solve's extra figures."""
    iters: int = 0
    rel_resid: float = float("nan")
    converged: bool = False
    status: str = ""
    true_rel_resid: float = float("nan")
    n_replacements: int = 0
    solve_ms: float = 0.0


# ---------------------------------------------------------------------------
# device context
# ---------------------------------------------------------------------------
class Context:
    """One iccg_ctx: a CUDA stream plus the device-resident system."""

    def __init__(self, device: int = 0):
        L = lib()
        h = C.c_void_p()
        _check(L.iccg_ctx_create(device, C.byref(h)))
        self.h = h
        self.n = 0
        self._sched_key = None

    def close(self):
        if getattr(self, "h", None):
            lib().iccg_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        _check(rc, self.h)

    @property
    def stream(self) -> int:
        return lib().iccg_ctx_stream(self.h) or 0

    @property
    def launches(self) -> int:
        return int(lib().iccg_ctx_launch_count(self.h))

    @property
    def device_bytes(self) -> int:
        return int(lib().iccg_ctx_device_bytes(self.h))

    def set_option(self, option: int, value: int):
        self._ck(lib().iccg_ctx_set_option(self.h, option, value))

    def use_tiled(self, on: bool):
        """Select the shared-memory tiled kernels (default) or the simple ones."""
        self.set_option(OPT_TILED, int(on))

    def upload(self, A: CRS):
        self._A = A
        self.n = A.n
        self._ck(lib().iccg_matrix_upload(self.h, A.n, _ptr(A.rowptr), _ptr(A.colind), _ptr(A.val)))
        self._sched_key = ("none",)

    def set_schedule(self, sched: Optional[ColorSchedule]):
        kind = 0 if sched is None else sched.kind()
        if kind == 0:
            key = ("none",)
        else:
            key = (id(sched), kind)
        if key == self._sched_key:
            return
        L = lib()
        if kind == 0:
            self._ck(L.iccg_schedule_none(self.h))
        elif kind == 1:
            cp, rc = _i32(sched.color_ptr), _i32(sched.rows_of_color)
            self._sched_arrays = (cp, rc)
            self._ck(L.iccg_schedule_mc(self.h, sched.nc, _ptr(cp), _ptr(rc)))
        else:
            arrs = tuple(_i32(a) for a in (sched.color_ptr_blk, sched.blocks_of_color, sched.block_ptr, sched.rows_of_block))
            self._sched_arrays = arrs
            self._ck(L.iccg_schedule_abmc(self.h, sched.nc, sched.nb, *[_ptr(a) for a in arrs]))
        self._sched_key = key

    def build(self, kind: int, shift: float = 0.0, auto_shift: bool = False):
        self._ck(lib().iccg_precond_build(self.h, kind, shift, int(auto_shift)))

    @property
    def shift(self) -> float:
        return float(lib().iccg_precond_shift(self.h))

    def apply(self, r: np.ndarray, storage: int = STORE_FP64) -> np.ndarray:
        r = _f64(r)
        z = np.zeros(self.n)
        self._ck(lib().iccg_precond_apply(self.h, _ptr(r), _ptr(z), storage))
        return z

    def spmv(self, x: np.ndarray, storage: int = STORE_FP64) -> np.ndarray:
        x = _f64(x)
        y = np.zeros(self.n)
        self._ck(lib().iccg_spmv(self.h, _ptr(x), _ptr(y), storage))
        return y

    def export_factor(self):
        L = lib()
        nnz = C.c_int()
        self._ck(L.iccg_precond_nnz(self.h, C.byref(nnz)))
        m = nnz.value
        Lp, Up = np.zeros(self.n + 1, np.int32), np.zeros(self.n + 1, np.int32)
        Li, Ui = np.zeros(m, np.int32), np.zeros(m, np.int32)
        Lx, Ux = np.zeros(m), np.zeros(m)
        self._ck(L.iccg_precond_export(self.h, _ptr(Lp), _ptr(Li), _ptr(Lx), _ptr(Up), _ptr(Ui), _ptr(Ux)))
        return Lp, Li, Lx, Up, Ui, Ux

    def solve(self, b: np.ndarray, x: np.ndarray, max_iter: int = 10000, tol: float = 1e-8,
              mode: int = MODE_FUSED, storage: int = STORE_FP64, rr_interval: int = 50,
              graph_iters: int = 16) -> CGResult:
        """conjugate_gradient on the uploaded A_run; x (float64, in/out)."""
        b = _f64(b)
        if x.dtype != np.float64 or not x.flags.c_contiguous:
            raise TypeError("x must be a contiguous float64 array (updated in place)")
        opts = _Opts(mode, storage, rr_interval, graph_iters)
        res = _Result()
        self._ck(lib().iccg_solve(self.h, _ptr(b), _ptr(x), int(max_iter), float(tol), C.byref(opts), C.byref(res)))
        return _cg_result(res)

    def solve_dev(self, b_ptr: int, x_ptr: int, max_iter: int = 10000, tol: float = 1e-8,
                  mode: int = MODE_FUSED, storage: int = STORE_FP64, rr_interval: int = 50,
                  graph_iters: int = 16) -> CGResult:
        """Same with device pointers (e.g. torch tensors' data_ptr())."""
        opts = _Opts(mode, storage, rr_interval, graph_iters)
        res = _Result()
        self._ck(lib().iccg_solve_dev(self.h, C.c_void_p(b_ptr), C.c_void_p(x_ptr), int(max_iter), float(tol),
                                      C.byref(opts), C.byref(res)))
        return _cg_result(res)

    def profile(self, enable: bool):
        self._ck(lib().iccg_profile_enable(self.h, int(enable)))

    def profile_read(self, cls: int):
        ms, n = C.c_double(), C.c_longlong()
        self._ck(lib().iccg_profile_read(self.h, cls, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    SWEEP_KINDS = ("chain", "staged", "two_phase", "one_phase", "csr", "persistent")

    def sweep_plan(self, storage: int = STORE_FP64, fwd: bool = True):
        """[(kind name, CTAs)] per level of the IC(0) sweep in that direction."""
        nl = C.c_int()
        self._ck(lib().iccg_sweep_plan(self.h, storage, int(fwd), None, None, 0, C.byref(nl)))
        kinds = np.zeros(max(nl.value, 1), np.int32)
        grids = np.zeros(max(nl.value, 1), np.int32)
        self._ck(lib().iccg_sweep_plan(self.h, storage, int(fwd), _ptr(kinds), _ptr(grids), nl.value, C.byref(nl)))
        return [(self.SWEEP_KINDS[k], int(g)) for k, g in zip(kinds[:nl.value], grids[:nl.value])]


def device_memory(device: int = 0):
    """(free, total) bytes of device memory (cudaMemGetInfo)."""
    f, t = C.c_longlong(), C.c_longlong()
    _check(lib().iccg_device_memory(int(device), C.byref(f), C.byref(t)))
    return f.value, t.value


class Batch:
    """Many independent solves advanced together (iccg_batch): one kernel
    launch per CG step for all of them.  Systems are Contexts with a matrix,
    a schedule and a built IC(0) preconditioner; each solve gives the bits,
    iterations and residuals of Context.solve on its system alone."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(lib().iccg_batch_create(device, C.byref(h)))
        self.h = h
        self.device = device
        self._systems: dict = {}      # index -> Context
        self._slot_n: dict = {}       # slot -> rows of its system

    def close(self):
        if getattr(self, "h", None):
            lib().iccg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        if rc != OK:
            raise IccgError(rc, lib().iccg_batch_last_error(self.h).decode(errors="replace"))

    def add_system(self, ctx: Context) -> int:
        """Adds a system (kept alive by the batch); returns its index."""
        idx = C.c_int()
        self._ck(lib().iccg_batch_add_system(self.h, ctx.h, C.byref(idx)))
        self._systems[idx.value] = ctx
        return idx.value

    def remove_system(self, index: int):
        """Takes out a system none of whose solves is in flight."""
        self._ck(lib().iccg_batch_remove_system(self.h, int(index)))
        self._systems.pop(int(index), None)

    def clear(self):
        self._ck(lib().iccg_batch_clear(self.h))
        self._systems = {}

    # -- continuous batching ------------------------------------------------
    def open(self, slots: int, storage: int = STORE_FP64, rr_interval: int = 50, graph_iters: int = 8):
        """Starts a session of `slots` solve slots (none may be in flight)."""
        self._ck(lib().iccg_batch_open(self.h, int(slots), C.byref(_Opts(MODE_FUSED, storage, rr_interval,
                                                                            graph_iters))))
        self._slot_n = {}

    def submit(self, system: int, b: np.ndarray, x0: Optional[np.ndarray] = None, max_iter: int = 10000,
               tol: float = 1e-8) -> int:
        """Admits a solve into a free slot (b and x0 are copied); returns the slot."""
        ctx = self._systems.get(int(system))
        if ctx is None:
            raise ValueError(f"no system {system}")
        b = _f64(b)
        if b.shape != (ctx.n,):
            raise ValueError(f"system {system} has {ctx.n} rows")
        if x0 is not None:
            x0 = _f64(x0)
            if x0.shape != (ctx.n,):
                raise ValueError(f"system {system} has {ctx.n} rows")
        slot = C.c_int()
        self._ck(lib().iccg_batch_submit(self.h, int(system), _ptr(b), _ptr(x0), int(max_iter), float(tol),
                                         C.byref(slot)))
        self._slot_n[slot.value] = ctx.n
        return slot.value

    def step(self, cap: int = 4096):
        """Advances every running solve graph_iters iterations; returns (slots
        that stopped, solves still running or waiting to start)."""
        out = np.zeros(max(1, cap), np.int32)
        ns, nr = C.c_int(), C.c_int()
        self._ck(lib().iccg_batch_step(self.h, _ptr(out), int(cap), C.byref(ns), C.byref(nr)))
        return [int(v) for v in out[:ns.value]], nr.value

    def retire(self, slots: Sequence[int]):
        """Solutions and results of stopped solves; frees their slots."""
        slots = [int(s) for s in slots]
        if not slots:
            return [], []
        xs = [np.zeros(self._slot_n[s]) for s in slots]
        sv = _i32(slots)
        xp = (C.c_void_p * len(slots))(*[x.ctypes.data for x in xs])
        res = (_Result * len(slots))()
        self._ck(lib().iccg_batch_retire(self.h, len(slots), _ptr(sv), xp, res))
        for s in slots:
            self._slot_n.pop(s, None)
        return xs, [_cg_result(r) for r in res]

    @property
    def launches(self) -> int:
        return int(lib().iccg_batch_launch_count(self.h))

    @property
    def device_bytes(self) -> int:
        return int(lib().iccg_batch_device_bytes(self.h))

    @property
    def device_ms(self) -> float:
        """Device time of the last solve() (CUDA events)."""
        return float(lib().iccg_batch_device_ms(self.h))

    def solve(self, systems: Sequence[int], bs: Sequence[np.ndarray], xs: Sequence[np.ndarray],
              max_iter: int = 10000, tol: float = 1e-8, storage: int = STORE_FP64, rr_interval: int = 50,
              graph_iters: int = 8) -> List[CGResult]:
        """Solve s: system systems[s], right-hand side bs[s], x0 / solution
        xs[s] (contiguous float64, updated in place)."""
        m = len(systems)
        if len(bs) != m or len(xs) != m:
            raise ValueError("systems, bs and xs differ in length")
        sysv = _i32(systems)
        bv = [_f64(b) for b in bs]
        for s, (k, b, x) in enumerate(zip(sysv, bv, xs)):
            if int(k) not in self._systems:
                raise ValueError(f"solve {s}: no system {k}")
            n = self._systems[int(k)].n
            if x.dtype != np.float64 or not x.flags.c_contiguous:
                raise TypeError("x must be a contiguous float64 array (updated in place)")
            if b.shape != (n,) or x.shape != (n,):
                raise ValueError(f"solve {s}: vectors of system {k} have {n} entries")
        bp = (C.c_void_p * m)(*[b.ctypes.data for b in bv])
        xp = (C.c_void_p * m)(*[x.ctypes.data for x in xs])
        res = (_Result * m)()
        opts = _Opts(MODE_FUSED, storage, rr_interval, graph_iters)
        self._ck(lib().iccg_batch_solve(self.h, m, _ptr(sysv), bp, xp, int(max_iter), float(tol), C.byref(opts),
                                        res))
        return [_cg_result(r) for r in res]


def _cg_result(res: _Result) -> CGResult:
    return CGResult(iters=res.iters, rel_resid=res.rel_resid, converged=bool(res.converged),
                    status=STATUS_NAMES.get(res.status, str(res.status)), true_rel_resid=res.true_rel_resid,
                    n_replacements=res.n_replacements, solve_ms=res.solve_ms)


# ---------------------------------------------------------------------------
# preconditioners with the reference's interface (precond.hpp, ic0.hpp)
# ---------------------------------------------------------------------------
class _GpuPrecond:
    kind = PRECOND_NONE

    def __init__(self, A: CRS, device: int = 0, storage: int = STORE_FP64):
        self.ctx = Context(device)
        self.ctx.upload(A)
        self.A = A
        self.storage = storage

    def apply(self, r, z, sched: Optional[ColorSchedule] = None):
        """z = M^{-1} r; z is resized/overwritten in place like the reference."""
        self.ctx.set_schedule(sched)
        out = self.ctx.apply(r, self.storage)
        if isinstance(z, np.ndarray):
            if z.shape != out.shape:
                z.resize(out.shape, refcheck=False)
            z[...] = out
        return out


class Identity(_GpuPrecond):
    """Identity (precond.hpp:8-17)."""
    kind = PRECOND_NONE

    def __init__(self, A: CRS, device: int = 0):
        super().__init__(A, device)
        self.ctx.build(PRECOND_NONE)

    def name(self) -> str:
        return "No preconditioner"


class Jacobi(_GpuPrecond):
    """Jacobi (precond.hpp:19-45)."""
    kind = PRECOND_JACOBI

    def __init__(self, A: CRS, device: int = 0):
        super().__init__(A, device)
        self.ctx.build(PRECOND_JACOBI)

    def name(self) -> str:
        return "Jacobi preconditioner"


class IC0(_GpuPrecond):
    """IC0 (ic0.hpp:11-76): IC(0) factor of A computed on the GPU.

    ``shift`` is added to every pivot as in the reference (ic0.cpp:103; the
    reference's default argument is 1e-12, its driver passes 0.0).  With
    ``auto_shift`` a non-positive pivot restarts the factorisation with a
    larger shift instead of raising.  ``sched`` may be given at construction
    so the factorisation runs in that schedule's parallel order.
    """
    kind = PRECOND_IC0

    def __init__(self, A: CRS, shift: float = 1e-12, device: int = 0, auto_shift: bool = False,
                 sched: Optional[ColorSchedule] = None):
        super().__init__(A, device)
        self.ctx.set_schedule(sched)
        self.ctx.build(PRECOND_IC0, shift, auto_shift)

    def name(self) -> str:
        return "IC preconditioner with multi-coloring"

    def factor(self):
        """(L_rowptr, L_colind, L_val, LT_colptr, LT_rowind, LT_val) of ic0.hpp:41-48."""
        return self.ctx.export_factor()


def conjugate_gradient(A: CRS, b, x, M: _GpuPrecond, max_iter: int, tol: float,
                       sched: Optional[ColorSchedule] = None, **opts) -> CGResult:
    """conjugate_gradient<Precond> (cg_crs.cpp:89-162) on the GPU.

    A must be the matrix M was built from; x is updated in place.  Keyword
    options: mode (MODE_FUSED / MODE_PLAIN), storage (STORE_FP64 /
    STORE_FP32), rr_interval, graph_iters.
    """
    if M.A is not A and (M.A.n != A.n or not np.array_equal(M.A.colind, A.colind)):
        raise ValueError("M was built from a different matrix")
    M.ctx.set_schedule(sched)
    opts.setdefault("storage", M.storage)
    return M.ctx.solve(b, x, max_iter, tol, **opts)
