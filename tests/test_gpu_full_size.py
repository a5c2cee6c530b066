"""The benchmark configurations at full size against the compiled reference
core (oracle/_ref/libfcaref_f32.so: the reference's src/common built with its
parity flags), FP32 bit for bit.

* config 2, 4096 x 4096 with the north-edge point inflow and 30 mm/h rain:
  the first 200 steps from the dry start, and 200 steps from the benchmark's
  warm start (20 mm on every cell, the state bench.py times);
* config 3, 2048 x 2048 with 100 mm/h rain for 3 h: the whole 6 h run.

Each runs with one, two and four columns per lane (the packed sweeps on
pairs of columns, one or two pairs per lane, on these all-LAND grids). The
reference core runs on every host core (OpenMP); 200 warm 4096^2 steps take
it about 20 s."""
import os

import numpy as np
import pytest

from floodca_b200 import synth
from floodca_b200.profile_step import warm_config2
from floodca_b200.sim import run_session
from oracle import refcore

pytestmark = [pytest.mark.gpu, pytest.mark.slow,
              pytest.mark.skipif(not refcore.available("f32"), reason="reference core not built")]


def _check(r, ref):
    assert r["step"] == ref["step"]
    assert r["t"] == ref["t"]
    for k in ("h", "hmax", "tmax"):
        assert np.array_equal(r[k], ref[k]), (k, float(np.abs(r[k] - ref[k]).max()))
    for k in ("V_rain", "V_bnd", "V_in", "clamp_err"):
        assert r[k] == pytest.approx(ref[k], rel=1e-9, abs=1e-6), k
    assert r["cap_active"] == ref["cap_active"]


def _threads():
    return os.cpu_count() or 1


@pytest.mark.parametrize("start", ["dry", "warm"])
def test_config2_full_size_equals_reference(start):
    d, p = synth.config2() if start == "dry" else warm_config2(4096)
    assert d.shape == (4096, 4096) and p.inflow_cell >= 0
    p = p.with_(steps=200)
    ref = refcore.run(d, p, kind="f32", threads=_threads())
    assert ref["V_in"] > 0.0
    for cpl in (1, 2, 4):
        _check(run_session(d, p, precision="f32", cols_per_lane=cpl), ref)


def test_config3_full_size_equals_reference():
    d, p = synth.config3()
    assert d.shape == (2048, 2048) and p.T_sim == 21600.0 and p.steps == 0
    ref = refcore.run(d, p, kind="f32", threads=_threads())     # the whole 6 h run
    assert ref["t"] == pytest.approx(p.T_sim) and ref["step"] > 1000
    for cpl in (1, 2, 4):
        _check(run_session(d, p, precision="f32", cols_per_lane=cpl), ref)
