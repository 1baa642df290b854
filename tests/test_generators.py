"""Synthetic workload generators, colorings and ABMC blockings."""
import numpy as np
import pytest

import iccg_b200 as ib
import iccg_b200.problems as pb


def _sym(A):
    D = A.to_dense()
    return np.array_equal(D, D.T)


def test_poisson2d_shape():
    A = pb.poisson2d(128)
    assert A.n == 16384 and A.nnz == 81408  # 5n - 4*128
    assert A.val[A.rowptr[200]:A.rowptr[201]].max() == 4.0


def test_laplace3d_aniso_shape():
    A = pb.laplace3d_aniso(8)
    assert A.n == 512 and A.nnz == 7 * 512 - 6 * 64
    assert _sym(A)
    d = A.to_dense()
    assert np.allclose(np.diag(d), 2 * (2 + 0.01))


@pytest.mark.slow
def test_config_sizes_full():
    A = pb.laplace3d_aniso(128)
    assert A.n == 2097152 and A.nnz == 14581760


def test_diffusion27():
    A = ib.gen_diffusion27(7, 6, 5, 1e4, 1)
    assert A.n == 210 and A.nnz == (3 * 7 - 2) * (3 * 6 - 2) * (3 * 5 - 2)
    D = A.to_dense()
    assert np.array_equal(D, D.T)
    off = D - np.diag(np.diag(D))
    assert (off <= 0).all()
    dd = np.diag(D) + off.sum(1)
    assert (dd >= -1e-12 * np.diag(D)).all()  # weakly diagonally dominant
    assert (dd > 1e-3 * np.diag(D)).any()     # strictly on the Dirichlet boundary
    assert np.linalg.eigvalsh(D).min() > 0


def test_diffusion27_contrast():
    A = ib.gen_diffusion27(12, 12, 12, 1e4, 2)
    # interior face couplings are harmonic means of kappa: their spread is
    # bounded by the 1e4 field contrast
    D = A.to_dense()
    c = -D[D < 0]
    assert c.max() / c.min() <= 1e4 * 4 + 1e-6


def test_knn_laplacian():
    A = ib.gen_knn_laplacian(500, 8, 1e-2, 3)
    D = A.to_dense()
    assert np.array_equal(D, D.T)
    assert np.allclose(D.sum(1), 1e-2)
    deg = (D != 0).sum(1) - 1
    assert deg.min() >= 8
    assert np.linalg.eigvalsh(D).min() > 0


def test_uniform_rng():
    x = ib.gen_uniform(100000, 0)
    assert x.min() >= -1 and x.max() < 1 and abs(x.mean()) < 0.01
    assert np.array_equal(x[:10], ib.gen_uniform(10, 0))


@pytest.mark.parametrize("make", [lambda: pb.poisson2d(20), lambda: pb.laplace3d_aniso(9),
                                  lambda: ib.gen_diffusion27(6, 6, 6, 100, 0), lambda: ib.gen_knn_laplacian(400, 8, 1e-2, 1)])
def test_greedy_coloring_is_proper(make):
    A = make()
    c, nc = ib.color_greedy(A)
    assert c.min() == 0 and c.max() == nc - 1
    for i in range(A.n):
        nbr = A.colind[A.rowptr[i]:A.rowptr[i + 1]]
        nbr = nbr[nbr != i]
        assert not np.any(c[nbr] == c[i])


@pytest.mark.parametrize("method", ["linear", "bfs"])
@pytest.mark.parametrize("B", [1, 8, 16, 33])
def test_abmc_blocking_valid(method, B):
    A = pb.laplace3d_aniso(9)
    blk, nb = ib.block_partition(A, B, method)
    counts = np.bincount(blk, minlength=nb)
    assert counts.max() <= B and counts.min() >= 1
    bcol, nc = ib.color_blocks(A, blk, nb)
    t, _ = ib.check_interblock_same_color(A, blk, bcol, nb, nc)
    assert t == 0
    P = pb.setup(A, "abmc", block_of_old=blk, nb=nb, block_color=bcol, nbc=nc)
    h, sb, xb = ib.check_schedule_hazards(P.A_run, P.new_of_old, P.color, P.block_of_old)
    assert xb == 0


def test_rhs_permuted():
    P = pb.make(pb.poisson2d(10), "piccg", seed=3)
    assert np.array_equal(P.b_run[P.new_of_old], P.b)
    assert np.allclose(P.A.to_dense() @ P.xstar, P.b)
