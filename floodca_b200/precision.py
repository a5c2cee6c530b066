"""Precision study (config 3: 2048 x 2048, three precisions) on the GPU.

The 2048 x 2048 config-1-generator grid (100 mm/h for 3 h, 6 h simulated)
runs three ways with the same kernel family:

  f32     FP32 stencil, FP64 volume / mass-balance accumulation and FP64
          simulated time (the reference float build's contract)
  f32all  FP32 everywhere, accumulators and simulated time included
  f64     FP64 everywhere (the reference FCA_DOUBLE build), the yardstick

and reports, against the FP64 run: max abs depth error (final depth and max
depth), RMSE of the max-depth map, wet-cell (h > 0.1 m) mismatches, and each
run's own mass-balance error.

    python -m floodca_b200.precision [--size 2048] [--out results.json]
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from . import synth
from .sim import run_session


def study(n: int = 2048, seed: int = 3) -> dict:
    dom, p = synth.config3(seed=seed, n=n)
    runs = {}
    for prec in ("f64", "f32", "f32all"):
        t0 = time.perf_counter()
        r = run_session(dom, p, precision=prec)
        r["wall_s"] = time.perf_counter() - t0
        runs[prec] = r
    ref = runs["f64"]
    out = {"workload": f"config 3: {n}x{n}, 90 m, fBm 5 m, 100 mm/h for 3 h, 6 h simulated",
           "cells": n * n, "runs": {}}
    wet_ref = np.asarray(ref["hmax"]) > 0.1
    for prec, r in runs.items():
        hm = np.asarray(r["hmax"], np.float64)
        hf = np.asarray(r["h"], np.float64)
        d_hmax = hm - np.asarray(ref["hmax"], np.float64)
        out["runs"][prec] = {
            "steps": r["step"], "t": r["t"], "wall_s": r["wall_s"],
            "max_abs_hmax_err_m": float(np.abs(d_hmax).max()),
            "rmse_hmax_m": float(np.sqrt(np.mean(d_hmax ** 2))),
            "max_abs_h_final_err_m": float(np.abs(hf - np.asarray(ref["h"], np.float64)).max()),
            "wet_mismatch_cells": int(((hm > 0.1) != wet_ref).sum()),
            "E_mass": r["E_mass"],
            "rel_volume_err_vs_f64": abs(r["V"] - ref["V"]) / max(ref["V"], 1e-30),
        }
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=2048)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--out", default="")
    a = ap.parse_args(argv)
    res = study(a.size, a.seed)
    txt = json.dumps(res, indent=1)
    if a.out:
        with open(a.out, "w") as f:
            f.write(txt + "\n")
    print(txt)
    return 0


if __name__ == "__main__":
    sys.exit(main())
