"""The reference's own CUDA-backend command-line driver (src/cuda/main_cuda.c
with src/common, unmodified, compiled by oracle/Makefile.ref) linked against
libfloodca_b200 in place of src/cuda/kernels.cu: it loads a grid directory
written by the synthetic generator, runs through fca_cuda_run and writes
hmax and h_final, which equal the reference's own CPU core (fca_run) on the
same grid: bit for bit in FP32, within 1e-12 m in FP64."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from floodca_b200 import synth
from floodca_b200.sim import RunParams
from oracle import refcore

pytestmark = pytest.mark.gpu
REF = Path(__file__).resolve().parents[1] / "oracle" / "_ref"


@pytest.mark.parametrize("kind,K,U", [("f32", 4, 1), ("f32", 8, 2), ("f64", 4, 1)])
def test_reference_cli_runs_on_the_dropin(tmp_path, kind, K, U):
    exe = REF / f"floodca_cuda_{kind}"
    if not exe.exists() or not refcore.available(kind):
        pytest.skip("the drop-in CLI and the reference core are built with the reference sources")
    d = synth.make_terrain(synth.TerrainSpec(90, 70, seed=9))
    d.h = np.full(d.shape, 0.01, np.float32)
    d.Rday = np.full(d.shape, 0.6, np.float32)          # 25 mm/h in m/day
    grid, out = tmp_path / "grid", tmp_path / "out"
    synth.write_grid_dir(d, grid)
    r = subprocess.run([str(exe), "--grid", str(grid), "--tsim", "3600", "--neigh", str(K),
                        "--U", str(U), "--hyeto", "uniform", "--out", str(out)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    done = [ln for ln in r.stdout.splitlines() if ln.startswith("done backend=cuda")]
    assert done, r.stdout
    steps = int(done[0].split("steps=")[1].split()[0])
    hmax = synth.read_field(out, "hmax", d.shape)
    h = synth.read_field(out, "h_final", d.shape)
    assert hmax.dtype == (np.float64 if kind == "f64" else np.float32)

    # the reference's CPU core on the grid as its loader reads it, with the
    # CLI's defaults (src/common/config.c) and the same options
    p = RunParams(K=K, U=U, hyeto="uniform", T_sim=3600.0)
    ref = refcore.run(synth.read_grid_dir(grid), p, kind=kind)
    assert steps == ref["step"] > 0
    if kind == "f32":
        assert np.array_equal(hmax, ref["hmax"]) and np.array_equal(h, ref["h"])
    else:
        # FP64: the double cube roots of CUDA and of glibc (the reference's
        # libm) are both faithfully rounded but may differ in the last bit
        for a, b in ((hmax, ref["hmax"]), (h, ref["h"])):
            assert np.abs(a - b).max() <= 1e-12

    # the Python API's session on the same grid writes the same output files
    from floodca_b200.sim import Session
    with Session(synth.read_grid_dir(grid), p, precision=kind) as sess:
        sess.run()
        sess.write_outputs(tmp_path / "mine")
    for name in ("hmax", "h_final"):
        mine = synth.read_field(tmp_path / "mine", name, d.shape)
        assert mine.dtype == hmax.dtype
        assert np.array_equal(mine, synth.read_field(out, name, d.shape)), name

