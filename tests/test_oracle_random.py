"""The oracle against the compiled reference core on seeded random small
grids (CPU): random sizes, relief, depths, Manning n, runoff, rain, SEA and
WALL cells; K = 4 / 8, U = 1..3, open or closed boundaries with random
per-edge flags, triangle or uniform hyetographs, fixed step counts or a
simulated time; FP32 and FP64. h, hmax, tmax, the step count and time must
be equal bit for bit. The golden fixtures pin chosen cases; this covers the
combinations between them."""
import numpy as np
import pytest

from floodca_b200 import abi
from floodca_b200.sim import Domain, RunParams
from oracle import pyoracle, refcore

pytestmark = pytest.mark.skipif(not refcore.available("f32") or not refcore.available("f64"),
                                reason="reference core not built")


def _case(seed):
    rng = np.random.default_rng(seed)
    nr, nc = int(rng.integers(1, 25)), int(rng.integers(1, 25))
    f = lambda lo, hi: rng.uniform(lo, hi, (nr, nc)).astype(np.float32)
    z = (f(0, 3) + np.linspace(2, 0, nr, dtype=np.float32)[:, None]).astype(np.float32)
    mask = np.zeros((nr, nc), np.uint8)
    u = rng.uniform(size=(nr, nc))
    mask[u < 0.08] = abi.FCA_SEA
    mask[(u >= 0.08) & (u < 0.14)] = abi.FCA_WALL
    h = f(0, 0.6) * (rng.uniform(size=(nr, nc)) < 0.7)
    dom = Domain(z=z, mask=mask, n=f(0.02, 0.15), C=f(0.2, 1.0), Rday=f(0.0, 0.4),
                 h=h.astype(np.float32), dx=float(rng.choice([10.0, 30.0, 90.0])))
    # bounded work: a fixed step count, or a short simulated time with
    # dt_min = 1 s (at most a few hundred steps). A fixed-step run keeps T_sim
    # out of reach: once t reaches T_sim the reference's loop takes dt = 0
    # steps forever (model.c:612-620 only stops a T_sim run).
    steps = int(rng.integers(5, 40)) if rng.uniform() < 0.6 else 0
    p = RunParams(K=int(rng.choice([4, 8])), U=int(rng.integers(1, 4)),
                  boundary="open" if rng.uniform() < 0.7 else "closed",
                  edges=tuple(int(x) for x in rng.integers(0, 2, 4)),
                  hyeto="uniform" if rng.uniform() < 0.5 else "triangle",
                  D_h=float(rng.uniform(0.05, 0.5)), phi=float(rng.uniform(0.1, 0.9)),
                  T_sim=float(rng.uniform(60, 400)) if steps == 0 else 1e6, steps=steps,
                  dt_min=1.0,
                  out_every=float(rng.choice([0.0, 90.0])))
    return dom, p


@pytest.mark.parametrize("kind", ["f32", "f64"])
@pytest.mark.parametrize("seed", range(100))
def test_oracle_equals_reference_random(seed, kind):
    dom, p = _case(1000 + seed)
    o = pyoracle.run(dom, p, double=(kind == "f64"))
    r = refcore.run(dom, p, kind=kind)
    assert o["step"] == r["step"] and o["t"] == r["t"], (o["step"], r["step"])
    for k in ("h", "hmax", "tmax"):
        assert np.array_equal(o[k], r[k]), k
