"""Same-box comparison with the reference's own CUDA backend.

The reference's command-line driver (src/cuda/main_cuda.c with src/common,
unmodified) is built twice by oracle/Makefile.ref: once on the reference's
CUDA backend (src/cuda/kernels.cu compiled for sm_100a with its release
flags, `floodca_cuda_ref`) and once on this repository's drop-in library
(`floodca_cuda_f32`). Both run the same grid directory (the warm config-2
terrain: 20 mm of water on every cell, 30 mm/h of rain) for the same fixed
step window, so the two `wall=` figures they print (the step loop of
fca_cuda_run, src/cuda/kernels.cu:712-732) compare the two backends on one
B200. The reference's float build contracts a*b+c into FMAs on the device,
so its depths differ from the exact ones by rounding only; both must agree
within the 1 mm parity bound.

Set FCAB_REFCUDA_SIZE to change the grid side (default 4096).
"""
import json
import os
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from floodca_b200 import synth
from floodca_b200.profile_step import warm_config2

pytestmark = pytest.mark.gpu
REF = Path(__file__).resolve().parents[1] / "oracle" / "_ref"
STEPS = 200


def _run(exe: Path, grid: Path, out: Path, cwd: Path) -> dict:
    r = subprocess.run([str(exe), "--grid", str(grid), "--steps", str(STEPS), "--hyeto",
                        "uniform", "--out", str(out)], capture_output=True, text=True,
                       timeout=600, cwd=cwd)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    done = [ln for ln in r.stdout.splitlines() if ln.startswith("done backend=cuda")]
    assert done, r.stdout[-2000:]
    f = dict(re.findall(r"(\w+)=(\S+)", done[0]))
    return {"steps": int(f["steps"]), "wall_s": float(f["wall"]), "h2d_s": float(f["h2d"]),
            "d2h_s": float(f["d2h"]), "E_mass": float(f["E_mass"]), "reduce": f["reduce"]}


def test_reference_cuda_backend_on_the_same_grid(tmp_path):
    ref_exe, mine_exe = REF / "floodca_cuda_ref", REF / "floodca_cuda_f32"
    if not ref_exe.exists() or not mine_exe.exists():
        pytest.skip("both CLIs are built with the reference sources (oracle/Makefile.ref)")
    n = int(os.environ.get("FCAB_REFCUDA_SIZE", "4096"))
    dom, _ = warm_config2(n)
    grid = tmp_path / "grid"
    synth.write_grid_dir(dom, grid)
    cells = int((dom.mask == 0).sum())
    res = {}
    for name, exe in (("reference_cuda", ref_exe), ("floodca_b200", mine_exe)):
        runs = [_run(exe, grid, tmp_path / name, tmp_path) for _ in range(2)]
        best = min(runs, key=lambda x: x["wall_s"])
        assert best["steps"] == STEPS
        best["gcells"] = cells * STEPS / best["wall_s"] / 1e9
        best["walls"] = [x["wall_s"] for x in runs]
        res[name] = best
    for field in ("hmax", "h_final"):
        a = synth.read_field(tmp_path / "reference_cuda", field, dom.shape).astype(np.float64)
        b = synth.read_field(tmp_path / "floodca_b200", field, dom.shape).astype(np.float64)
        assert np.abs(a - b).max() <= 1e-3, field
        res.setdefault("max_abs_diff_m", {})[field] = float(np.abs(a - b).max())
    res["grid"] = [n, n]
    res["steps"] = STEPS
    res["speedup"] = res["floodca_b200"]["gcells"] / res["reference_cuda"]["gcells"]
    print("REFCUDA " + json.dumps(res))
