"""Land cover to Manning n and runoff coefficient C.

The engine reads n and C as rasters; this module makes them from an ESA
WorldCover class raster the way the reference's data preparation does
(FloodCA prep/floodca_prep/landcover.py:35-70 and config/landcover_params.csv):

  * a table maps each WorldCover code to (manning_n, runoff_C); codes absent
    from the table take the row with code -1 (0.035, 0.40 when the table has
    none);
  * n is scaled by k_n, C by k_C and clipped to [0, 1], in float32;
  * for a 90 m grid made from a 30 m class raster, n and C are the float32
    means of each 3 x 3 block (C clipped to [0, 1] again) and the class is the
    block's most frequent code (the smallest code on a tie).

`load_table` reads a table file with the reference's columns
(worldcover_code, class, manning_n, runoff_C); WORLDCOVER holds the values of
the reference's table, for runs without the file.
"""
from __future__ import annotations

import csv
from pathlib import Path

import numpy as np

from .sim import Domain

# WorldCover code -> (Manning n, runoff C), the classes of the reference's
# config/landcover_params.csv; -1 is the default row
WORLDCOVER: dict[int, tuple[float, float]] = {
    10: (0.12, 0.20),     # tree cover
    20: (0.07, 0.30),     # shrubland
    30: (0.035, 0.35),    # grassland
    40: (0.04, 0.35),     # cropland
    50: (0.015, 0.85),    # built-up
    60: (0.025, 0.60),    # bare / sparse vegetation
    70: (0.02, 0.90),     # snow and ice
    80: (0.03, 1.00),     # permanent water bodies
    90: (0.06, 0.10),     # herbaceous wetland
    95: (0.12, 0.10),     # mangroves
    100: (0.035, 0.30),   # moss and lichen
    -1: (0.035, 0.40),    # default
}
DEFAULT_ROW = (0.035, 0.40)


def load_table(path) -> dict[int, tuple[float, float]]:
    """Reads a land-cover table (columns worldcover_code, manning_n, runoff_C)."""
    table: dict[int, tuple[float, float]] = {}
    with Path(path).open("r", encoding="utf-8") as f:
        for row in csv.DictReader(f):
            table[int(row["worldcover_code"])] = (float(row["manning_n"]), float(row["runoff_C"]))
    return table


def lookup(lc: np.ndarray, table: dict[int, tuple[float, float]] | None = None,
           k_n: float = 1.0, k_c: float = 1.0) -> tuple[np.ndarray, np.ndarray]:
    """(n, C) float32 rasters of the class raster `lc`."""
    table = WORLDCOVER if table is None else table
    default = table.get(-1, DEFAULT_ROW)
    codes = np.unique(lc)
    n_of = np.array([table.get(int(c), default)[0] for c in codes], np.float32)
    c_of = np.array([table.get(int(c), default)[1] for c in codes], np.float32)
    idx = np.searchsorted(codes, lc)
    n = n_of[idx]
    C = c_of[idx]
    n *= np.float32(k_n)
    C = np.clip(C * np.float32(k_c), np.float32(0.0), np.float32(1.0))
    return n.astype(np.float32), C.astype(np.float32)


def block_majority_3(lc: np.ndarray) -> np.ndarray:
    """Most frequent code of each 3 x 3 block (smallest code on a tie)."""
    h, w = lc.shape
    x = lc.reshape(h // 3, 3, w // 3, 3).transpose(0, 2, 1, 3).reshape(h // 3, w // 3, 9)
    codes, inv = np.unique(x, return_inverse=True)
    inv = inv.reshape(h // 3, w // 3, 9)
    counts = np.zeros((h // 3, w // 3, len(codes)), np.int32)
    for i in range(len(codes)):
        counts[..., i] = (inv == i).sum(axis=2)
    return codes[counts.argmax(axis=-1)].astype(lc.dtype)


def block_mean_3(a: np.ndarray) -> np.ndarray:
    """float32 mean of each 3 x 3 block."""
    h, w = a.shape
    return a.reshape(h // 3, 3, w // 3, 3).mean(axis=(1, 3)).astype(np.float32)


def lookup_90m(lc30: np.ndarray, table=None, k_n: float = 1.0, k_c: float = 1.0):
    """A 90 m grid's (class, n, C) from a 30 m class raster (sides multiples
    of 3)."""
    n30, c30 = lookup(lc30, table, k_n, k_c)
    return (block_majority_3(lc30), block_mean_3(n30),
            np.clip(block_mean_3(c30), np.float32(0.0), np.float32(1.0)))


def apply(dom: Domain, lc: np.ndarray, table=None, k_n: float = 1.0, k_c: float = 1.0) -> Domain:
    """A copy of `dom` whose n and C come from the class raster `lc` (same
    shape as the grid)."""
    if lc.shape != dom.shape:
        raise ValueError(f"class raster {lc.shape} does not match the grid {dom.shape}")
    out = dom.copy()
    out.n, out.C = lookup(lc, table, k_n, k_c)
    return out
