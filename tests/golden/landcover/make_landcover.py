"""Generates worldcover.npz (this directory) from the FloodCA reference's own
land-cover lookup (prep/floodca_prep/landcover.py: load_lc_table,
_lookup_n_c, _agg_majority_3, _agg_mean_3) and table
(config/landcover_params.csv).

The reference module imports rasterio, which this environment lacks, so the
four functions are taken out of the module's syntax tree and executed with
numpy and csv only; nothing else of the module runs.

Run from the repository root where the reference sources exist:
    python tests/golden/landcover/make_landcover.py --ref /path/to/floodca
"""
from __future__ import annotations

import argparse
import ast
import csv
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
FUNCS = ("load_lc_table", "_lookup_n_c", "_agg_majority_3", "_agg_mean_3")


def reference_functions(ref: Path) -> dict:
    src = (ref / "prep" / "floodca_prep" / "landcover.py").read_text()
    tree = ast.parse(src)
    body = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in FUNCS]
    mod = ast.Module(body=body, type_ignores=[])
    ns = {"np": np, "csv": csv, "Path": Path}
    exec(compile(ast.fix_missing_locations(mod), "landcover.py", "exec"), ns)
    return {k: ns[k] for k in FUNCS}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True)
    a = ap.parse_args()
    ref = Path(a.ref)
    f = reference_functions(ref)
    table = f["load_lc_table"](ref / "config" / "landcover_params.csv")
    rng = np.random.default_rng(17)
    codes = np.array([0, 10, 20, 30, 40, 50, 60, 70, 80, 90, 95, 100, 255], np.uint8)
    lc30 = codes[rng.integers(0, len(codes), (48, 63))]
    lc30[:9, :9] = 40                                   # uniform blocks
    lc30[9:12, :3] = np.array([[10, 10, 20], [20, 30, 30], [40, 50, 60]], np.uint8)  # a tie
    out = {"lc30": lc30,
           "table_codes": np.array(sorted(table), np.int64),
           "table_n": np.array([table[c][0] for c in sorted(table)], np.float64),
           "table_C": np.array([table[c][1] for c in sorted(table)], np.float64)}
    for tag, (k_n, k_c) in {"k1": (1.0, 1.0), "k2": (1.3, 1.6), "k3": (0.7, 0.5)}.items():
        n30, c30 = f["_lookup_n_c"](lc30, table, k_n, k_c)
        out[f"{tag}_kn_kc"] = np.array([k_n, k_c])
        out[f"{tag}_n30"], out[f"{tag}_c30"] = n30, c30
        out[f"{tag}_lc90"] = f["_agg_majority_3"](lc30)
        out[f"{tag}_n90"] = f["_agg_mean_3"](n30)
        out[f"{tag}_c90"] = np.clip(f["_agg_mean_3"](c30), 0.0, 1.0)
    np.savez_compressed(HERE / "worldcover.npz", **out)
    print("wrote", HERE / "worldcover.npz")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
