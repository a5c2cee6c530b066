"""The C oracle restatement reproduces the reference's own outputs (the
golden fixtures made by the compiled reference core) bit for bit."""
import numpy as np
import pytest

from conftest import GOLDEN, golden_cases
from tests.golden.make_golden import load_case
from oracle import pyoracle

ACC_EXACT = ("step", "cap_active", "cap_total", "dt_min_hits", "t", "dt_base")
ACC_CLOSE = ("V", "V0", "V_rain", "V_sea", "V_bnd", "clamp_err", "V_in")


@pytest.mark.parametrize("kind", ["f32", "f64"])
@pytest.mark.parametrize("case", golden_cases())
def test_oracle_matches_reference(case, kind):
    d, p, f, force = load_case(GOLDEN / f"{case}.npz")
    r = pyoracle.run(d, p, double=(kind == "f64"), force_rday=force)
    for k in ("h", "hmax", "tmax"):
        assert np.array_equal(r[k], f[f"{kind}_{k}"]), f"{case}/{kind}: {k} differs"
    acc = f[f"{kind}_acc"]
    for k in ACC_EXACT:
        assert r[k] == pytest.approx(acc[k], rel=0, abs=0), k
    for k in ACC_CLOSE:
        # double sums in a different (threaded) order
        assert r[k] == pytest.approx(acc[k], rel=1e-12, abs=1e-9), k
