"""The caller's PtAP + lower-to-full expansion on the device
(iccg_ptap_full_gpu) against the host routines (themselves bit-exact with the
reference's Permute_PtAP_LowerCRS_to_LowerCRS and expand_lower_to_full): the
same rows, columns and value bits, on stencils, the 27-point operator, kNN
graphs, explicit zeros (dropped), unsymmetric lower values, a 1x1 system;
inputs that repeat an (i, j) pair, or give long rows, go to the host routines
with the same result; bad input is rejected."""
import time

import numpy as np
import pytest

import iccg_b200 as ib
import iccg_b200.problems as pb

pytestmark = pytest.mark.gpu


def _host(A, p):
    return ib.expand_lower_to_full(ib.Permute_PtAP_LowerCRS_to_LowerCRS(A, p))


def _same(a, b):
    assert a.n == b.n
    assert np.array_equal(a.rowptr, b.rowptr)
    assert np.array_equal(a.colind, b.colind)
    assert np.array_equal(a.val.view(np.uint64), b.val.view(np.uint64))


def _perm(n, seed):
    return np.random.default_rng(seed).permutation(n).astype(np.int32)


@pytest.mark.parametrize("which", ["p2d", "l3d", "d27", "knn", "abmc_perm"])
def test_gpu_ptap_full_matches_host(which):
    if which == "abmc_perm":
        P = pb.config_abmc_aniso(20, 16, "bfs", seed=1)
        A, p = P.A, P.new_of_old
    else:
        A = {"p2d": lambda: pb.poisson2d(50), "l3d": lambda: pb.laplace3d_aniso(14),
             "d27": lambda: ib.gen_diffusion27(12, 12, 12, 1e4, 3), "knn": lambda: ib.gen_knn_laplacian(4000, 8, 1e-2, 5)}[which]()
        p = _perm(A.n, 7)
    B, on_dev = ib.Permute_PtAP_full_gpu(A, p)
    assert on_dev
    _same(B, _host(A, p))


def test_gpu_ptap_full_drops_zeros_and_reads_only_the_lower_triangle():
    A = pb.laplace3d_aniso(8)
    val = A.val.copy()
    rng = np.random.default_rng(3)
    # explicit zeros (one of them on a diagonal) and upper values that differ
    # from their mirrors: the lower triangle alone decides the result
    lower = np.concatenate([np.arange(A.rowptr[i], A.rowptr[i + 1])[A.colind[A.rowptr[i]:A.rowptr[i + 1]] <= i]
                            for i in range(A.n)])
    val[rng.choice(lower, 40, replace=False)] = 0.0
    upper = np.setdiff1d(np.arange(A.nnz), lower)
    val[upper] *= 1.0 + rng.standard_normal(upper.size) * 1e-3
    A2 = ib.CRS(A.n, A.rowptr, A.colind, val)
    p = _perm(A.n, 11)
    B, on_dev = ib.Permute_PtAP_full_gpu(A2, p)
    assert on_dev
    _same(B, _host(A2, p))
    assert B.nnz < A.nnz


def test_gpu_ptap_full_hands_repeated_pairs_to_the_host():
    # row 2 holds column 1 twice: the sum depends on the order
    rp = np.array([0, 1, 3, 6], np.int32)
    ci = np.array([0, 0, 1, 1, 1, 2], np.int32)
    v = np.array([4.0, -1.0, 4.0, 0.1, 0.2, 4.0])
    A = ib.CRS(3, rp, ci, v)
    p = np.array([2, 0, 1], np.int32)
    B, on_dev = ib.Permute_PtAP_full_gpu(A, p)
    assert not on_dev
    _same(B, _host(A, p))
    one = ib.CRS(1, np.array([0, 1], np.int32), np.array([0], np.int32), np.array([2.0]))
    B, on_dev = ib.Permute_PtAP_full_gpu(one, np.array([0], np.int32))
    _same(B, _host(one, np.array([0], np.int32)))


def test_gpu_ptap_full_rejects_bad_input():
    A = pb.poisson2d(6)
    with pytest.raises(ib.IccgError):
        ib.Permute_PtAP_full_gpu(A, np.zeros(A.n, np.int32))          # not a permutation
    bad = A.colind.copy()
    bad[5] = A.n + 3
    with pytest.raises(ib.IccgError):
        ib.Permute_PtAP_full_gpu(ib.CRS(A.n, A.rowptr, bad, A.val), _perm(A.n, 1))


@pytest.mark.slow
def test_gpu_ptap_full_at_the_benchmark_size():
    """The 128^3 system as bench.py builds it: device against host, and the
    two timings (printed)."""
    P = pb.config_abmc_aniso(128, 16, "linear", seed=0)
    t0 = time.perf_counter()
    B, on_dev = ib.Permute_PtAP_full_gpu(P.A, P.new_of_old)
    t1 = time.perf_counter()
    H = _host(P.A, P.new_of_old)
    t2 = time.perf_counter()
    assert on_dev
    _same(B, H)
    _same(B, P.A_run)
    print(f"ptap+expand 128^3: device {1e3 * (t1 - t0):.1f} ms, host {1e3 * (t2 - t1):.1f} ms")
