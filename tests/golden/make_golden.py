"""Generates the golden fixtures in this directory from the FloodCA reference.

The reference ships no test vectors, so the fixtures are produced by the
reference itself: its core (src/common/*.c, compiled from the sources in
place by oracle/Makefile.ref into oracle/_ref/) runs each case through
oracle/refcore.py, in the FP32 parity build (-ffp-contract=off) and the
FCA_DOUBLE build. Each case file <name>.npz holds the inputs, the run
parameters (JSON), and the reference outputs h, hmax, tmax plus the run
accumulators, for both precisions.

Run from the repository root where the reference sources exist:
    python tests/golden/make_golden.py [--ref /path/to/floodca]
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from floodca_b200 import synth  # noqa: E402
from floodca_b200.sim import Domain, RunParams  # noqa: E402
from oracle import refcore  # noqa: E402

ACC_KEYS = ("V", "V0", "V_rain", "V_sea", "V_bnd", "clamp_err", "cap_active", "cap_total",
            "dt_min_hits", "t", "step", "dt_base", "V_in", "E_mass")


def terrain(nr, nc, seed, amp=5.0):
    return synth.make_terrain(synth.TerrainSpec(nr, nc, amplitude=amp, seed=seed))


def case_c1_64():
    return synth.config1(n=64, seed=11)


def _mixed(seed):
    rng = np.random.default_rng(seed)
    d = terrain(40, 56, seed)
    # SEA in the south-west corner at sea level, a WALL ridge, spatial C/Rday
    d.mask[30:, :12] = 1
    d.z[30:, :12] = 0.0
    d.mask[10, 20:35] = 2
    d.mask[5:9, 44] = 2
    d.C = rng.uniform(0.2, 1.0, d.shape).astype(np.float32)
    d.Rday = rng.uniform(0.05, 0.4, d.shape).astype(np.float32)
    h = np.zeros(d.shape, np.float32)
    h[12:20, 25:40] = rng.uniform(0.0, 0.8, (8, 15)).astype(np.float32)
    d.h = h
    return d


def case_mixed_k4():
    d = _mixed(21)
    p = RunParams(K=4, U=1, boundary="open", hyeto="triangle", D_h=2.0, phi=0.4,
                  T_sim=3 * 3600.0, z_sea=0.0)
    return d, p


def case_mixed_k8():
    d = _mixed(22)
    p = RunParams(K=8, U=3, boundary="closed", hyeto="uniform", steps=300, T_sim=86400.0)
    return d, p


def case_mixed_k8_open():
    d = _mixed(23)
    p = RunParams(K=8, U=1, boundary="open", edges=(1, 0, 1, 1), hyeto="triangle", D_h=1.0,
                  phi=0.5, T_sim=5400.0, out_every=900.0)
    return d, p


def case_inflow():
    d, p = synth.box_rain(terrain(48, 48, 31, amp=3.0), synth.south_open(), 20.0, 0.5)
    p = p.with_(T_sim=5400.0, inflow_cell=24, inflow_peak=50.0, inflow_t_peak=1800.0,
                inflow_t_end=3600.0)
    return d, p


def case_lambda():
    d, p = synth.box_rain(terrain(24, 30, 41), RunParams(boundary="open"), 40.0, 2.0)
    return d, p.with_(lambda_=1.7, T_sim=4000.0, rain_end=0.0, U=2)


def _tiny(nr, nc, seed):
    rng = np.random.default_rng(seed)
    d = terrain(max(nr, 2), max(nc, 2), seed)
    sl = (slice(0, nr), slice(0, nc))
    d = Domain(z=d.z[sl].copy(), mask=d.mask[sl].copy(), n=d.n[sl].copy(), C=d.C[sl].copy(),
               Rday=np.full((nr, nc), 0.3, np.float32), h=rng.uniform(0, 0.5, (nr, nc)).astype(np.float32),
               dx=30.0)
    p = RunParams(boundary="open", hyeto="uniform", T_sim=1800.0)
    return d, p


def case_tiny_1x1():
    return _tiny(1, 1, 51)


def case_tiny_1x7():
    return _tiny(1, 7, 52)


def case_tiny_7x1():
    return _tiny(7, 1, 53)


def case_tiny_3x3():
    return _tiny(3, 3, 54)


def case_tiny_2x5():
    d, p = _tiny(2, 5, 55)
    return d, p.with_(K=8)


def _column(k):
    n = 64
    z = np.full((n, n), 10.0, np.float32)
    h = np.zeros((n, n), np.float32)
    h[n // 2 - 2:n // 2 + 3, n // 2 - 2:n // 2 + 3] = 1.0
    d = Domain(z=z, mask=np.zeros((n, n), np.uint8), n=np.full((n, n), 0.03, np.float32),
               C=np.zeros((n, n), np.float32), Rday=np.zeros((n, n), np.float32), h=h, dx=90.0)
    return d, RunParams(K=k, U=1, boundary="closed", steps=400)


def case_column_k4():
    return _column(4)


def case_column_k8():
    return _column(8)


def case_forcing():
    d = terrain(16, 20, 61)
    rng = np.random.default_rng(61)
    days = [rng.uniform(0.0, 0.2, d.shape).astype(np.float32) for _ in range(2)]
    p = RunParams(boundary="open", edges=(0, 1, 0, 0), hyeto="uniform", T_sim=1.25 * 86400.0,
                  out_every=3600.0)
    return d, p, days


CASES = {
    "c1_64": case_c1_64, "mixed_k4": case_mixed_k4, "mixed_k8": case_mixed_k8,
    "mixed_k8_open": case_mixed_k8_open, "inflow": case_inflow, "lambda": case_lambda,
    "tiny_1x1": case_tiny_1x1, "tiny_1x7": case_tiny_1x7, "tiny_7x1": case_tiny_7x1,
    "tiny_3x3": case_tiny_3x3, "tiny_2x5": case_tiny_2x5, "column_k4": case_column_k4,
    "column_k8": case_column_k8, "forcing": case_forcing,
}


# The isotropy protocol of the reference's analysis/e9_aniso.py, reduced: a
# flat plane at 90 m, closed, no rain, a 5x5 column of 1 m, runs of CHUNK
# steps each restarted from the float32 depth (hmax = h, t = 0), FP64.
E9_SMALL = {"n": 512, "chunk": 400, "chunks": 30, "thresh": 1e-3}


def e9_domain(n):
    z = np.full((n, n), 10.0, np.float32)
    h = np.zeros((n, n), np.float32)
    c = n // 2
    h[c - 2:c + 3, c - 2:c + 3] = 1.0
    return Domain(z=z, mask=np.zeros((n, n), np.uint8), n=np.full((n, n), 0.03, np.float32),
                  C=np.zeros((n, n), np.float32), Rday=np.zeros((n, n), np.float32), h=h, dx=90.0)


def make_e9_small(K):
    """Wet-cell counts after every chunk and the final float32 depth, from
    the reference core in FP64."""
    n, chunk = E9_SMALL["n"], E9_SMALL["chunk"]
    d = e9_domain(n)
    p = RunParams(K=K, U=1, boundary="closed", steps=chunk)
    h32 = d.h.copy()
    wet = []
    for _ in range(E9_SMALL["chunks"]):
        dd = Domain(z=d.z, mask=d.mask, n=d.n, C=d.C, Rday=d.Rday, h=h32, dx=d.dx)
        r = refcore.run(dd, p, "f64")
        h32 = np.asarray(r["h"], np.float64).astype(np.float32)
        wet.append(int((np.asarray(r["h"], np.float64) > E9_SMALL["thresh"]).sum()))
    return {"wet": np.asarray(wet, np.int64), "h_final": h32, "K": np.int64(K),
            "params": json.dumps(E9_SMALL)}


def write_forcing(days, tmp: Path) -> list[str]:
    files = []
    for i, r in enumerate(days):
        f = tmp / f"rday_{i}.bin"
        np.asarray(r, np.float32).tofile(f)
        files.append(str(f))
    return files


def make_case(name: str) -> dict:
    made = CASES[name]()
    days = None
    if len(made) == 3:
        d, p, days = made
    else:
        d, p = made
    out = {"params": json.dumps(dataclasses.asdict(p)), "dx": np.float64(d.dx)}
    for k in ("z", "mask", "n", "C", "Rday", "h"):
        out[f"in_{k}"] = getattr(d, k)
    if days is not None:
        out["in_force_rday"] = np.stack(days)
    for kind in ("f32", "f64"):
        with tempfile.TemporaryDirectory() as tmp:
            ff = write_forcing(days, Path(tmp)) if days is not None else None
            r = refcore.run(d, p, kind, force_files=ff)
        for k in ("h", "hmax", "tmax"):
            out[f"{kind}_{k}"] = r[k]
        out[f"{kind}_acc"] = json.dumps({k: float(r[k]) for k in ACC_KEYS})
    return out


def load_case(path: Path):
    """Returns (Domain, RunParams, fixture dict, force_rday or None)."""
    f = dict(np.load(path, allow_pickle=False))
    pd = json.loads(str(f["params"]))
    pd["edges"] = tuple(pd["edges"])
    p = RunParams(**pd)
    d = Domain(z=f["in_z"], mask=f["in_mask"], n=f["in_n"], C=f["in_C"], Rday=f["in_Rday"],
               h=f["in_h"], dx=float(f["dx"]))
    for kind in ("f32", "f64"):
        f[f"{kind}_acc"] = json.loads(str(f[f"{kind}_acc"]))
    return d, p, f, f.get("in_force_rday")


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("cases", nargs="*")
    a = ap.parse_args()
    if not refcore.build(a.ref):
        print(f"reference sources not found under {a.ref}", file=sys.stderr)
        return 1
    for name in [c for c in (a.cases or CASES) if c in CASES]:
        np.savez_compressed(HERE / f"{name}.npz", **make_case(name))
        print("wrote", name)
    if not a.cases or "e9" in a.cases:
        for K in (4, 8):
            np.savez_compressed(HERE / f"e9_small_k{K}.npz", **make_e9_small(K))
            print("wrote e9_small", K)
    # ABI layout of the reference structs, from oracle/_ref/abi_probe_*
    import subprocess
    layout = {k: json.loads(subprocess.check_output([str(refcore.REF_DIR / f"abi_probe_{k}")]))
              for k in ("f32", "f64")}
    (HERE / "abi_layout.json").write_text(json.dumps(layout, indent=1) + "\n")
    # The reference's published isotropy experiment (analysis/e9_aniso.py,
    # results/e9_anisotropy.json): a known answer for a long closed run.
    e9 = json.loads(Path(a.ref, "results/e9_anisotropy.json").read_text())
    (HERE / "e9_reference.json").write_text(json.dumps(
        {"source": "results/e9_anisotropy.json", **e9}, indent=1) + "\n")
    print("wrote abi_layout.json, e9_reference.json")
    return 0


if __name__ == "__main__":
    sys.exit(main())
