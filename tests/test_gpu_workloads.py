"""The benchmark workloads on the GPU against the oracle at sizes the oracle
finishes in seconds, and size-independent properties at full size."""
import numpy as np
import pytest

from floodca_b200 import synth
from floodca_b200.sim import Session, run_session
from oracle import pyoracle

pytestmark = pytest.mark.gpu


def _diff(a, b):
    return float(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max())


@pytest.mark.parametrize("kind", ["f32", "f64"])
def test_config1_full_size_matches_oracle(kind):
    d, p = synth.config1()
    r = run_session(d, p, precision=kind)
    o = pyoracle.run(d, p, double=(kind == "f64"))
    assert r["step"] == o["step"]
    assert _diff(r["h"], o["h"]) <= 1e-6 and _diff(r["hmax"], o["hmax"]) <= 1e-6
    assert abs(r["V"] - o["V"]) / o["V"] < 1e-9


def test_config2_shape_with_inflow_matches_oracle():
    d, p = synth.config2(n=512)
    p = p.with_(T_sim=3 * 3600.0)
    r = run_session(d, p, precision="f32")
    o = pyoracle.run(d, p)
    assert r["step"] == o["step"]
    assert _diff(r["hmax"], o["hmax"]) <= 1e-6
    assert r["V_in"] == pytest.approx(o["V_in"], rel=1e-12)
    assert abs(r["V"] - o["V"]) / o["V"] < 1e-9


def test_config3_shape_precision_variants():
    d, p = synth.config3(n=256)
    p = p.with_(T_sim=2 * 3600.0)
    r32 = run_session(d, p, precision="f32")
    r64 = run_session(d, p, precision="f64")
    rall = run_session(d, p, precision="f32all")
    o = pyoracle.run(d, p)
    assert _diff(r32["hmax"], o["hmax"]) <= 1e-6
    # FP32 against FP64: within the 1 mm bar on this case, mass balance tight
    assert _diff(r32["hmax"], r64["hmax"]) < 1e-3
    assert r32["E_mass"] < 1e-6 and r64["E_mass"] < 1e-12
    assert _diff(rall["hmax"], r64["hmax"]) < 1e-2


@pytest.mark.parametrize("cpl", [1, 2, 4])
def test_fast_math_within_tolerance(cpl):
    """Hardware approximations against the exact run, on the scalar sweep
    (one column per lane) and the packed sweeps (two and four)."""
    d, p = synth.config1()
    ex = run_session(d, p, precision="f32", math="exact", cols_per_lane=cpl)
    fa = run_session(d, p, precision="f32", math="fast", cols_per_lane=cpl)
    assert _diff(ex["hmax"], fa["hmax"]) <= 1e-3
    assert abs(ex["V"] - fa["V"]) / ex["V"] <= 1e-5


@pytest.mark.parametrize("cpl", [2, 4])
def test_fp32_everywhere_packed_sweeps_equal_scalar(cpl):
    """FP32-everywhere (float time and volume accumulators) on the packed
    sweeps equals the scalar sweep in the same precision: depths, maxima,
    times and steps bit for bit, volumes within float rounding (the
    accumulation order differs)."""
    d, p = synth.config1()
    r1 = run_session(d, p, precision="f32all", cols_per_lane=1)
    rp = run_session(d, p, precision="f32all", cols_per_lane=cpl)
    assert rp["step"] == r1["step"] and rp["t"] == r1["t"]
    for k in ("h", "hmax", "tmax"):
        assert np.array_equal(rp[k], r1[k]), k
    for k in ("V", "V_rain", "V_bnd"):
        assert rp[k] == pytest.approx(r1[k], rel=1e-4, abs=1e-3), k


def test_tma_row_source_equals_reference(monkeypatch):
    """The pair sweep's TMA row source (FCAB_ROW_SOURCE=tma: z, h, n rows
    through a shared-memory ring filled by cp.async.bulk.tensor) gives the
    reference core's results bit for bit, like the plain loads."""
    from floodca_b200.profile_step import warm_config2
    from tests import refpin
    d, p = warm_config2(512)
    p = p.with_(steps=120)
    monkeypatch.setenv("FCAB_ROW_SOURCE", "tma")
    with Session(d, p, precision="f32", cols_per_lane=2) as s:
        assert s.info()["tma_rows"] == 1
        s.run()
        st = s.stats()
        h, hmax, tmax = s.download()
    refpin.check_reference({"h": h, "hmax": hmax, "tmax": tmax, **st}, d, p)


def test_config2_full_size_properties():
    """4096^2 run for 30 simulated minutes: mass balance, non-negative
    depth, hmax >= h, and the inflow volume matches its closed form."""
    d, p = synth.config2()
    p = p.with_(T_sim=1800.0)
    r = run_session(d, p, precision="f32")
    assert r["E_mass"] < 1e-5
    assert (r["h"] >= 0).all() and (r["hmax"] >= r["h"]).all()
    tp = 3 * 3600.0
    want = 0.5 * 500.0 * (1800.0 / tp) * 1800.0
    assert r["V_in"] == pytest.approx(want, rel=1e-9)
