"""Seeded synthetic domains standing in for the reference's rasters.

The reference's real grids (Udupi 90 m rasters) are not shipped, so every
workload is generated: a plane sloping toward the south edge (row nrows-1),
plus fractional-Brownian-motion relief, plus a carved north-south channel,
with six land-cover classes laid out as Voronoi patches. Manning n comes
from the class; runoff coefficient C = 1; every cell is LAND unless a
caller adds SEA or WALL cells.

Relief: spectral synthesis with power ~ k^-(2H+2) (H = Hurst exponent),
random phases, normalised so its values span [-amplitude, +amplitude].
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .sim import Domain, RunParams

MANNING_CLASSES = (0.02, 0.035, 0.05, 0.07, 0.10, 0.15)


def fbm(nr: int, nc: int, hurst: float, amplitude: float, rng: np.random.Generator) -> np.ndarray:
    ky = np.fft.fftfreq(nr)[:, None]
    kx = np.fft.rfftfreq(nc)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    k[0, 0] = 1.0
    amp = k ** (-(hurst + 1.0))          # |F| ~ k^-(H+1)  <=>  power ~ k^-(2H+2)
    amp[0, 0] = 0.0
    phase = rng.uniform(0.0, 2.0 * np.pi, size=amp.shape)
    spec = amp * np.exp(1j * phase)
    f = np.fft.irfft2(spec, s=(nr, nc))
    f -= f.mean()
    span = np.abs(f).max()
    return f * (amplitude / span) if span > 0 else f


def voronoi_classes(nr: int, nc: int, n_classes: int, rng: np.random.Generator,
                    cells_per_patch: int = 4096) -> np.ndarray:
    """Class index per cell from the nearest of a set of random seed points."""
    from scipy.spatial import cKDTree
    nseed = max(8, (nr * nc) // cells_per_patch)
    pts = np.column_stack([rng.uniform(0, nr, nseed), rng.uniform(0, nc, nseed)])
    cls = rng.integers(0, n_classes, nseed)
    tree = cKDTree(pts)
    out = np.empty((nr, nc), np.int8)
    cc = np.arange(nc) + 0.5
    step = max(1, (1 << 22) // nc)
    for r0 in range(0, nr, step):
        r1 = min(nr, r0 + step)
        rr = (np.arange(r0, r1) + 0.5)[:, None]
        q = np.column_stack([np.repeat(rr, nc, axis=1).ravel(), np.tile(cc, r1 - r0)])
        _, idx = tree.query(q)
        out[r0:r1] = cls[idx].reshape(r1 - r0, nc)
    return out


@dataclass
class TerrainSpec:
    nrows: int
    ncols: int
    dx: float = 90.0
    slope: float = 0.005           # fall per metre toward the south edge
    hurst: float = 0.7
    amplitude: float = 5.0         # relief spans [-amplitude, +amplitude] m
    channel_width: int = 3
    channel_depth: float = 2.0
    base: float = 10.0             # elevation of the south edge, m
    seed: int = 1
    n_scale: float = 1.0           # multiplies every class's Manning n


def make_terrain(spec: TerrainSpec) -> Domain:
    rng = np.random.default_rng(spec.seed)
    nr, nc = spec.nrows, spec.ncols
    rows = np.arange(nr, dtype=np.float64)[:, None]
    z = spec.base + spec.slope * spec.dx * (nr - 1 - rows) + np.zeros((1, nc))
    z = z + fbm(nr, nc, spec.hurst, spec.amplitude, rng)
    c0 = nc // 2 - spec.channel_width // 2
    z[:, c0:c0 + spec.channel_width] -= spec.channel_depth
    cls = voronoi_classes(nr, nc, len(MANNING_CLASSES), rng)
    n = np.asarray(MANNING_CLASSES, np.float64)[cls] * spec.n_scale
    zero = np.zeros((nr, nc), np.float32)
    return Domain(z=z.astype(np.float32), mask=np.zeros((nr, nc), np.uint8),
                  n=n.astype(np.float32), C=np.ones((nr, nc), np.float32), Rday=zero.copy(),
                  h=zero.copy(), dx=spec.dx)


def box_rain(dom: Domain, p: RunParams, mm_per_h: float, hours: float) -> tuple[Domain, RunParams]:
    """Uniform rain of mm_per_h for `hours` from t = 0: a uniform hyetograph
    (F = dt/86400 per step) with Rday in m/day, C = 1, and the rain switched
    off at rain_end."""
    d = dom.copy()
    d.Rday = np.full(d.shape, mm_per_h * 24.0 / 1000.0, np.float32)
    d.C = np.ones(d.shape, np.float32)
    return d, p.with_(hyeto="uniform", rain_end=hours * 3600.0)


# ---------------------------------------------------------------------------
# The workloads (sizes, forcing and durations of the benchmark configurations).

def south_open() -> RunParams:
    """Open south edge, other edges closed; 10-minute output windows
    (out_every = 600 s), so steps also land on every rain end that is a
    multiple of 10 minutes, which the reference can then represent."""
    return RunParams(boundary="open", edges=(0, 1, 0, 0), out_every=600.0)


def config1(seed: int = 1, n: int = 256) -> tuple[Domain, RunParams]:
    """256x256, 90 m, fBm 5 m, 50 mm/h for 1 h, open south, 2 h simulated."""
    dom = make_terrain(TerrainSpec(n, n, amplitude=5.0, seed=seed))
    return box_rain(dom, south_open().with_(T_sim=7200.0), 50.0, 1.0)


def config2(seed: int = 2, n: int = 4096) -> tuple[Domain, RunParams]:
    """4096x4096, fBm 20 m, north-edge point inflow (0 -> 500 m^3/s at 3 h -> 0 at
    6 h, symmetric triangle), 30 mm/h for 2 h, open south, 6 h simulated."""
    dom = make_terrain(TerrainSpec(n, n, amplitude=20.0, seed=seed))
    dom, p = box_rain(dom, south_open().with_(T_sim=21600.0), 30.0, 2.0)
    p = p.with_(inflow_cell=0 * n + n // 2, inflow_peak=500.0, inflow_t_peak=3 * 3600.0,
                inflow_t_end=6 * 3600.0)
    return dom, p


def config3(seed: int = 3, n: int = 2048) -> tuple[Domain, RunParams]:
    """2048x2048 from the config-1 generator, 100 mm/h for 3 h, 6 h simulated."""
    dom = make_terrain(TerrainSpec(n, n, amplitude=5.0, seed=seed))
    return box_rain(dom, south_open().with_(T_sim=21600.0), 100.0, 3.0)
