"""Step-control helpers of the oracle (hyetograph integral, next event,
point inflow) against the reference and against closed forms."""
import ctypes as C
import math

import numpy as np
import pytest

from floodca_b200.sim import RunParams
from oracle import pyoracle, refcore
from floodca_b200 import synth


def _params(**kw):
    d = synth.make_terrain(synth.TerrainSpec(4, 4))
    return d, RunParams(**kw)


def test_triangle_hyetograph_integrates_to_one():
    d, p = _params(hyeto="triangle", D_h=6.0, phi=0.3)
    q = pyoracle.params_of(d, p)
    L = pyoracle.lib(False)
    tot = sum(L.or_hyeto_integral(C.byref(q), t, 37.0) for t in np.arange(0, 6 * 3600 + 37, 37.0))
    assert tot == pytest.approx(1.0, rel=1e-12)


def test_uniform_hyetograph_is_dt_over_day():
    d, p = _params(hyeto="uniform")
    q = pyoracle.params_of(d, p)
    assert pyoracle.lib(False).or_hyeto_integral(C.byref(q), 100.0, 43.2) == 43.2 / 86400.0


@pytest.mark.parametrize("t", [0.0, 599.9999999999, 600.0, 86399.0, 86400.0, 1234.5])
def test_next_event_matches_reference(t):
    d, p = _params(out_every=600.0, T_sim=2 * 86400.0)
    q = pyoracle.params_of(d, p)
    r = refcore.RefRun(d, p, "f32")
    assert pyoracle.lib(False).or_next_event_time(C.byref(q), t) == \
        r.L.fca_next_event_time(C.byref(r.cfg), t)


def test_rain_end_is_an_event():
    d, p = _params(rain_end=1000.0, T_sim=5000.0)
    q = pyoracle.params_of(d, p)
    L = pyoracle.lib(False)
    assert L.or_next_event_time(C.byref(q), 10.0) == 1000.0
    assert L.or_next_event_time(C.byref(q), 1000.0) == 5000.0


def test_inflow_volume_total_and_split():
    d, p = _params(inflow_cell=0, inflow_peak=500.0, inflow_t_peak=3 * 3600.0,
                   inflow_t_end=6 * 3600.0)
    q = pyoracle.params_of(d, p)
    L = pyoracle.lib(False)
    tot = sum(L.or_inflow_volume(C.byref(q), t, 53.0) for t in np.arange(0, 6 * 3600 + 53, 53.0))
    assert tot == pytest.approx(0.5 * 500.0 * 6 * 3600.0, rel=1e-12)
    for t, dt in ((100.0, 17.0), (10790.0, 20.0), (21590.0, 30.0)):
        assert L.or_inflow_volume(C.byref(q), t, dt) == pytest.approx(
            refcore.inflow_volume(p, t, dt), rel=1e-15)


def test_cbrt_sq_is_double_cube_root_rounded():
    L = pyoracle.lib(False)
    for x in (1e-3, 0.0123, 1.0, 2.5, 777.0):
        xf = np.float32(x)
        want = np.float32(math.pow(float(xf) * float(xf), 1.0 / 3.0))
        assert abs(L.or_cbrt_sq(float(xf)) - float(want)) <= 1.2e-7 * float(want)
