"""Shared helpers of the test suite."""
from __future__ import annotations

from pathlib import Path
from types import SimpleNamespace

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def golden_names():
    return sorted(p.stem for p in GOLDEN.glob("*.npz"))


def load_golden(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


def golden_sched(g: dict):
    """ColorSchedule-like namespace from a fixture (None for cg/dcg/iccg)."""
    v = str(g["variant"])
    if v == "piccg":
        return SimpleNamespace(nc=int(g["nc"]), color_ptr=g["color_ptr"], rows_of_color=g["rows_of_color"], mode=0,
                               nb=0, color_ptr_blk=None, blocks_of_color=None, block_ptr=None, rows_of_block=None)
    if v == "abmc":
        return SimpleNamespace(nc=int(g["nc"]), color_ptr=None, rows_of_color=None, mode=1, nb=int(g["nb"]),
                               color_ptr_blk=g["color_ptr_blk"], blocks_of_color=g["blocks_of_color"],
                               block_ptr=g["block_ptr"], rows_of_block=g["rows_of_block"])
    return None


def to_color_schedule(s):
    import iccg_b200 as ib
    if s is None:
        return None
    return ib.ColorSchedule(nc=s.nc, color_ptr=s.color_ptr, rows_of_color=s.rows_of_color, mode=s.mode, nb=s.nb,
                            color_ptr_blk=s.color_ptr_blk, blocks_of_color=s.blocks_of_color,
                            block_ptr=s.block_ptr, rows_of_block=s.rows_of_block)


def rel_err(x, y) -> float:
    x, y = np.asarray(x), np.asarray(y)
    d = np.linalg.norm(y)
    return float(np.linalg.norm(x - y) / (d if d > 0 else 1.0))
