"""The CUDA sessions against the compiled reference core on the seeded random
small grids that pin the oracle (tests/test_oracle_random.py): random sizes,
relief, depths, Manning n, runoff, rain, SEA and WALL cells; K = 4 / 8,
U = 1..3, open or closed boundaries with random per-edge flags, triangle or
uniform hyetographs, fixed step counts or a simulated time.

Each grid also runs as an all-LAND grid (SEA and WALL cells turned to LAND),
which takes the all-LAND kernels, with the random C*Rday field as a per-cell
rain field. Every lane width runs: one column per lane, two (the packed
pair sweep on all-LAND grids) and four (two pairs per lane on all-LAND K = 4
grids). FP32 must equal the reference bit for bit;
FP64 depths within 1e-12 m and times within 1e-9 s (the device's and glibc's
double cube roots may differ in the last bit)."""
import numpy as np
import pytest

from floodca_b200.sim import run_session
from oracle import refcore
from tests.test_oracle_random import _case

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refcore.available("f32") or not refcore.available("f64"),
                                 reason="reference core not built")]


def _check(r, ref, kind):
    assert r["step"] == ref["step"], (r["step"], ref["step"])
    if kind == "f32":
        assert r["t"] == ref["t"]
    else:
        assert r["t"] == pytest.approx(ref["t"], abs=1e-9)
    for k in ("h", "hmax", "tmax"):
        if kind == "f32":
            assert np.array_equal(r[k], ref[k]), k
        else:
            # depths within 1e-12 m; tmax holds times (seconds), which carry
            # the clock's last-bit differences, within the same 1e-9 s as t
            tol = 1e-9 if k == "tmax" else 1e-12
            assert np.abs(np.asarray(r[k], np.float64) - ref[k]).max() <= tol, k
    for k in ("V_rain", "V_sea", "V_bnd", "clamp_err"):
        assert r[k] == pytest.approx(ref[k], rel=1e-9, abs=1e-6), k
    assert r["cap_active"] == ref["cap_active"]


@pytest.mark.parametrize("kind", ["f32", "f64"])
@pytest.mark.parametrize("seed", range(100))
def test_session_equals_reference_random(seed, kind):
    dom, p = _case(1000 + seed)
    ref = refcore.run(dom, p, kind=kind)
    for cpl in (1, 2, 4):
        _check(run_session(dom, p, precision=kind, cols_per_lane=cpl), ref, kind)


@pytest.mark.parametrize("seed", range(100))
def test_all_land_session_equals_reference_random(seed):
    dom, p = _case(1000 + seed)
    dom = dom.copy()
    dom.mask[:] = 0
    ref = refcore.run(dom, p, kind="f32")
    for cpl in (1, 2, 4):
        _check(run_session(dom, p, precision="f32", cols_per_lane=cpl), ref, "f32")
