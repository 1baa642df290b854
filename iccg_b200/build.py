"""Build recipe for the iccg_b200 shared library (sm_100a) and the oracle.

``python -m iccg_b200.build`` compiles every CUDA and C++ source of the
package with nvcc into ``iccg_b200/_lib/libiccg_b200.so`` (in-tree, so the
library travels with the repository), and runs ``make -C oracle`` to build
the test oracle.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "_lib"
LIB = LIBDIR / "libiccg_b200.so"

CUDA_SOURCES = ["ctx.cu", "noalloc.cu", "setup_dev.cu"]
HOST_SOURCES = ["host_order.cpp", "host_gen.cpp", "host_layout.cpp", "host_capi.cpp"]
HEADERS = ["dd.cuh", "kernels.cuh", "persist.cuh", "host.hpp", "devbuf.hpp", "context.hpp", "plan.inl", "factor.inl",
           "qsys.inl", "persist.inl", "solver.inl", "batch.inl"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    # explicit fma() only: the reference's rounding is reproduced by hand
    "--fmad=false",
    "-Xcompiler", "-fPIC,-O3,-march=x86-64-v3,-ffp-contract=off",
    "-shared",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _host_cxx() -> str | None:
    # nvcc's host compiler; the environment may point CXX at a wrapper
    for cand in ("/usr/bin/g++",):
        if Path(cand).exists():
            return cand
    return None


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build_library(force: bool = False, verbose: bool = False) -> Path:
    deps = [CSRC / s for s in CUDA_SOURCES + HOST_SOURCES + HEADERS] + [ROOT / "include" / "iccg.h"]
    if not force and not _stale(LIB, deps):
        return LIB
    LIBDIR.mkdir(exist_ok=True)
    cmd = [_nvcc(), *NVCC_FLAGS]
    cxx = _host_cxx()
    if cxx:
        cmd += ["-ccbin", cxx]
    cmd += [str(CSRC / s) for s in CUDA_SOURCES + HOST_SOURCES]
    cmd += ["-o", str(LIB), "--cudart=static"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


def build_oracle(verbose: bool = False) -> None:
    make = shutil.which("make")
    if make is None:
        raise RuntimeError("make not found")
    out = subprocess.run([make, "-C", str(ROOT / "oracle")], capture_output=not verbose, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + (out.stdout or "") + (out.stderr or ""))


def main(argv: list[str]) -> int:
    force = "--force" in argv
    build_library(force=force, verbose=True)
    build_oracle(verbose=True)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
