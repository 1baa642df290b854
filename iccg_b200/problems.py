"""Problem set-up: the driver steps of the reference's main() and the
synthetic workloads the solver is measured on.

``setup(A, variant, ...)`` replays cg_crs.cpp:386-484 with this package's
bit-exact host routines: read colors or blocks, build new_of_old, form
A_run = P^T A P (lower-only, then expanded to full) and the ColorSchedule.
``variant`` names the reference binary (Makefile:18-53): ``cg`` (Identity),
``dcg`` (Jacobi), ``iccg`` (IC(0), natural order), ``piccg`` (IC(0) + MC),
``abmc`` (IC(0) + ABMC).

The workloads stand in for the SuiteSparse matrix of the reference's scripts
(run_*.sh), which is not available: seeded stencils, a variable-coefficient
27-point diffusion operator and k-NN graph Laplacians, each with
b = A x*, x* ~ U(-1,1) from splitmix64.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import (CRS, ColorSchedule, BuildABMCSchedule, BuildColorPtrRows_FromPermutationAndColor,
               BuildPermutationByBlockColor, BuildPermutationByColor, Permute_PtAP_LowerCRS_to_LowerCRS,
               Permute_PtAP_full_gpu,
               block_partition, color_blocks, color_greedy, expand_lower_to_full, gen_diffusion27,
               gen_knn_laplacian, gen_stencil_2d5, gen_stencil_3d7, gen_uniform, host_spmv)

VARIANTS = ("cg", "dcg", "iccg", "piccg", "abmc")

# device on which setup() forms A_run (iccg_ptap_full_gpu: the same bits as
# the host routines), or None for the host routines
PTAP_DEVICE: Optional[int] = None


@dataclass
class Problem:
    name: str
    variant: str
    A: CRS                          # original order (what the reader returns)
    A_run: CRS                      # the matrix CG runs on (cg_crs.cpp:442-447)
    sched: Optional[ColorSchedule]  # None for cg / dcg / iccg
    new_of_old: Optional[np.ndarray] = None
    color: Optional[np.ndarray] = None       # node colors (old ids)
    nc: int = 0
    block_of_old: Optional[np.ndarray] = None
    block_color: Optional[np.ndarray] = None
    nb: int = 0
    xstar: Optional[np.ndarray] = None       # original order
    b: Optional[np.ndarray] = None           # original order
    b_run: Optional[np.ndarray] = None       # permuted
    info: dict = field(default_factory=dict)

    @property
    def precond_kind(self) -> int:
        return {"cg": 0, "dcg": 1}.get(self.variant, 2)

    def unpermute(self, x_run: np.ndarray) -> np.ndarray:
        if self.new_of_old is None:
            return x_run
        return x_run[self.new_of_old]


def setup(A: CRS, variant: str, color=None, nc: int = 0, block_of_old=None, nb: int = 0, block_color=None,
          nbc: int = 0, name: str = "") -> Problem:
    """cg_crs.cpp:386-484 for one variant."""
    if variant not in VARIANTS:
        raise ValueError(f"variant must be one of {VARIANTS}")
    P = Problem(name=name, variant=variant, A=A, A_run=A, sched=None)
    if variant == "piccg":
        color = np.ascontiguousarray(color, np.int32)
        new_of_old = BuildPermutationByColor(color)
        P.color, P.nc = color, int(nc)
    elif variant == "abmc":
        block_of_old = np.ascontiguousarray(block_of_old, np.int32)
        block_color = np.ascontiguousarray(block_color, np.int32)
        color = block_color[block_of_old]                     # cg_crs.cpp:406-408
        new_of_old = BuildPermutationByBlockColor(block_of_old, block_color)
        P.color, P.nc = color, int(nbc)
        P.block_of_old, P.block_color, P.nb = block_of_old, block_color, int(nb)
    else:
        return P
    P.new_of_old = new_of_old
    if PTAP_DEVICE is not None:
        P.A_run, _ = Permute_PtAP_full_gpu(A, new_of_old, PTAP_DEVICE)   # cg_crs.cpp:419-421 on the GPU
    else:
        Ap = Permute_PtAP_LowerCRS_to_LowerCRS(A, new_of_old)
        P.A_run = expand_lower_to_full(Ap)                     # cg_crs.cpp:420-421
    if variant == "abmc":
        cpb, boc, bp, rob = BuildABMCSchedule(new_of_old, block_of_old, block_color, nb, nbc)
        P.sched = ColorSchedule(nc=nbc, mode=ColorSchedule.ABMC_BLOCK, nb=nb, color_ptr_blk=cpb,
                                blocks_of_color=boc, block_ptr=bp, rows_of_block=rob)
        cp, rc = BuildColorPtrRows_FromPermutationAndColor(color, nbc, new_of_old)
        P.sched.color_ptr, P.sched.rows_of_color = cp, rc
    else:
        cp, rc = BuildColorPtrRows_FromPermutationAndColor(color, nc, new_of_old)
        P.sched = ColorSchedule(nc=nc, color_ptr=cp, rows_of_color=rc)
    return P


def with_rhs(P: Problem, seed: int = 0) -> Problem:
    """b = A x*, x* ~ U(-1,1) from splitmix64(seed), in the original order and
    permuted to the run order (b_run[new_of_old[i]] = b[i])."""
    P.xstar = gen_uniform(P.A.n, seed)
    P.b = host_spmv(P.A, P.xstar)
    if P.new_of_old is None:
        P.b_run = P.b.copy()
    else:
        P.b_run = np.empty_like(P.b)
        P.b_run[P.new_of_old] = P.b
    return P


def make(A: CRS, variant: str, block_size: int = 16, blocking: str = "bfs", seed: int = 0, name: str = "") -> Problem:
    """Colors / blocks from this package's generators, then setup()."""
    if variant == "piccg":
        color, nc = color_greedy(A)
        P = setup(A, variant, color=color, nc=nc, name=name)
    elif variant == "abmc":
        blk, nb = block_partition(A, block_size, blocking)
        bcol, nbc = color_blocks(A, blk, nb)
        P = setup(A, variant, block_of_old=blk, nb=nb, block_color=bcol, nbc=nbc, name=name)
        P.info["block_size"] = block_size
        P.info["blocking"] = blocking
    else:
        P = setup(A, variant, name=name)
    return with_rhs(P, seed)


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------
def poisson2d(side: int = 128) -> CRS:
    """2D 5-point Poisson, side x side interior grid, Dirichlet (diag 4, off -1)."""
    return gen_stencil_2d5(side, side)


def laplace3d_aniso(side: int = 128, wz: float = 0.01) -> CRS:
    """3D 7-point Laplacian, side^3, coefficients 1, 1, wz (diag 2(2+wz))."""
    return gen_stencil_3d7(side, side, side, 1.0, 1.0, wz)


def config_small_mc(side: int = 128, seed: int = 0) -> Problem:
    """Plain FP64 multicolor ICCG on the 2D 5-point Poisson problem, greedy
    coloring, b = A x* (seed 0)."""
    return make(poisson2d(side), "piccg", seed=seed, name=f"poisson2d_{side}_mc")


def config_abmc_aniso(side: int = 128, block_size: int = 16, blocking: str = "bfs", seed: int = 0) -> Problem:
    """ABMC ICCG on the anisotropic 3D 7-point Laplacian (1, 1, 0.01)."""
    return make(laplace3d_aniso(side), "abmc", block_size=block_size, blocking=blocking, seed=seed,
                name=f"laplace3d_aniso_{side}_abmc{block_size}")


def config_diffusion27(side: int = 96, variant: str = "abmc", block_size: int = 16, seed: int = 0,
                       contrast: float = 1e4) -> Problem:
    """27-point variable-coefficient diffusion (log-normal, 1e4 contrast)."""
    A = gen_diffusion27(side, side, side, contrast, seed)
    return make(A, variant, block_size=block_size, seed=seed, name=f"diffusion27_{side}_{variant}{block_size}")


def config_knn(npts: int, seed: int = 0, block_size: int = 16) -> Problem:
    """Symmetrised 8-NN graph Laplacian + 1e-2 I on npts points."""
    A = gen_knn_laplacian(npts, 8, 1e-2, seed)
    return make(A, "abmc", block_size=block_size, seed=seed, name=f"knn_{npts}")
