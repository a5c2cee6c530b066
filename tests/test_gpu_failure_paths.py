"""Failure paths through the reference-facing fca_cuda_run on the device.

* A forcing day whose file is missing, short or unnamed ends the run where
  that day begins, as the reference's loop does (src/cuda/kernels.cu:497-507
  and 712-732): acc.t is set to T_sim and the state is the state of the
  steps taken before the failed load (checked against a fixed-step run of
  the same forcing with every file present). Unlike the reference, which
  returns 0 there, fca_cuda_run returns -3, so a caller such as the
  reference's CLI does not take the truncated run for a complete one.
* A non-finite z, h, n, C or Rday on a LAND cell makes the upload fail:
  fca_cuda_run returns -2 and fcab_last_error names the field and the cell.
  The reference does not check its inputs; non-finite values would spread
  through the depths without an error. The model never reads n, C or Rday
  off LAND nor z or h of SEA cells, so non-finite values there are accepted
  and change nothing.
* After each failure the library stays usable: a following good run gives
  the reference's golden result.
"""
import tempfile
from pathlib import Path

import numpy as np
import pytest

from conftest import GOLDEN
from floodca_b200 import abi, lib
from floodca_b200.sim import DropinGrid
from tests.golden.make_golden import load_case

pytestmark = pytest.mark.gpu


def _forcing_grid(tmp, force, files=None, steps=0):
    d, p, f, _ = load_case(GOLDEN / "forcing.npz")
    g = DropinGrid(d, p)
    paths = []
    for i, r in enumerate(force):
        path = Path(tmp) / f"rday_{i}.bin"
        np.asarray(r, np.float32).tofile(path)
        paths.append(path)
    for i, path in enumerate(files if files is not None else paths):
        g.cfg.force_files[i].value = str(path).encode()
    g.cfg.n_force_days = len(force)
    g.cfg.hyeto = abi.FCA_HYETO_UNIFORM
    g.cfg.steps = steps
    return g, f


def _golden_run_ok():
    """The forcing golden case, all files present, equals the reference."""
    _, _, _, force = load_case(GOLDEN / "forcing.npz")
    with tempfile.TemporaryDirectory() as tmp:
        g, f = _forcing_grid(tmp, force)
        assert g.run() == 0
    r = g.result()
    assert r["step"] == f["f32_acc"]["step"]
    assert np.array_equal(r["h"], f["f32_h"])


@pytest.mark.parametrize("how", ["missing", "short", "empty_name"])
def test_failed_forcing_day_ends_the_run_and_is_reported(how):
    _, p, _, force = load_case(GOLDEN / "forcing.npz")
    assert len(force) == 2 and p.T_sim > 86400.0
    with tempfile.TemporaryDirectory() as tmp:
        day1 = Path(tmp) / "day1.bin"
        if how == "short":
            np.asarray(force[1], np.float32).ravel()[:-1].tofile(day1)
        files = [str(Path(tmp) / "rday_0.bin"), "" if how == "empty_name" else str(day1)]
        g, _ = _forcing_grid(tmp, force, files=files)
        assert g.run() == -3
        r = g.result()
        assert r["t"] == p.T_sim                      # the reference's end marker
        n = r["step"]
        assert n > 0
        # the same steps with every file present, by step count
        good, _ = _forcing_grid(tmp, force, steps=n)
        assert good.run() == 0
        rg = good.result()
    assert rg["step"] == n and rg["t"] >= 86400.0 and rg["t"] < p.T_sim
    for k in ("h", "hmax", "tmax"):
        assert np.array_equal(r[k], rg[k]), k
    _golden_run_ok()


@pytest.mark.parametrize("field", ["z", "h", "n", "C", "Rday"])
@pytest.mark.parametrize("value", [np.nan, np.inf])
def test_non_finite_land_input_is_rejected(field, value):
    d, p, f, _ = load_case(GOLDEN / "mixed_k4.npz")
    g = DropinGrid(d.copy(), p)          # the grid may share the domain's arrays
    land = np.flatnonzero(d.mask.ravel() == abi.FCA_LAND)
    cell = int(land[len(land) // 2])
    g.arrays[field].reshape(-1)[cell] = value
    assert g.run() == -2
    msg = lib.core().fcab_last_error().decode()
    r, c = divmod(cell, d.shape[1])
    assert f"{field} is not finite at LAND cell (row {r}, col {c})" in msg, msg
    # the library is still usable
    g2 = DropinGrid(d, p)
    assert g2.run() == 0
    res = g2.result()
    assert np.array_equal(res["h"], f["f32_h"])


def test_non_finite_values_off_land_are_ignored():
    """n, C and Rday of SEA and WALL cells and z, h of SEA cells are never
    read (physics.h:64-100: a WALL face carries nothing, a SEA cell's level
    is z_sea with no depth and its faces take the LAND side's n); a WALL
    cell's z is its level in the slope of the dt pass, so it is left alone."""
    d, p, f, _ = load_case(GOLDEN / "mixed_k4.npz")
    m = d.mask.ravel()
    off = np.flatnonzero(m != abi.FCA_LAND)
    sea = np.flatnonzero(m == abi.FCA_SEA)
    assert off.size > 0 and sea.size > 0
    g = DropinGrid(d.copy(), p)
    for k in ("n", "C", "Rday"):
        g.arrays[k].reshape(-1)[off] = np.nan
    for k in ("z", "h"):
        g.arrays[k].reshape(-1)[sea] = np.nan
    assert g.run() == 0
    r = g.result()
    land = d.mask == abi.FCA_LAND
    assert np.array_equal(r["h"][land], f["f32_h"][land])
    assert r["step"] == f["f32_acc"]["step"]
