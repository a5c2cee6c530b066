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


# ---------------------------------------------------------------------------
# The reference's grid directory (FloodCA src/common/grid.c:162-237,
# src/common/io.c:34-56): dem.json {nrows, ncols, dx, dtype, x0, y0, ...}
# and raw row-major float32 rasters dem.bin, n.bin, C.bin, Rday.bin, h.bin
# plus uint8 mask.bin (row 0 = north). Missing optional rasters load as
# n = 0.03, C = 0, Rday = 0, h = 0.

def write_grid_dir(dom: Domain, path, name: str = "synthetic", x0: float = 0.0,
                   y0: float = 0.0) -> None:
    """Writes `dom` as a grid directory the reference's CLIs read (--grid)."""
    import json
    from pathlib import Path
    d = Path(path)
    d.mkdir(parents=True, exist_ok=True)
    nr, nc = dom.shape
    hdr = {"name": name, "nrows": int(nr), "ncols": int(nc), "dx": float(dom.dx),
           "dtype": "float32", "crs": "EPSG:32643", "x0": float(x0), "y0": float(y0),
           "nodata": -9999, "source": "floodca_b200.synth", "sha256": ""}
    (d / "dem.json").write_text(json.dumps(hdr) + "\n")
    for fname, arr in (("dem", dom.z), ("n", dom.n), ("C", dom.C), ("Rday", dom.Rday),
                       ("h", dom.h)):
        np.ascontiguousarray(arr, np.float32).tofile(d / f"{fname}.bin")
    np.ascontiguousarray(dom.mask, np.uint8).tofile(d / "mask.bin")


def read_grid_dir(path) -> Domain:
    """Reads a grid directory as the reference's fca_grid_load_dir does."""
    import json
    from pathlib import Path
    d = Path(path)
    hdr = json.loads((d / "dem.json").read_text())
    nr, nc, dx = int(hdr["nrows"]), int(hdr["ncols"]), float(hdr.get("dx", 30.0))

    def f32(name, default):
        p = d / f"{name}.bin"
        if p.exists():
            return np.fromfile(p, np.float32, nr * nc).reshape(nr, nc)
        return np.full((nr, nc), default, np.float32)

    h = f32("h", None) if (d / "h.bin").exists() else f32("h0", 0.0)
    return Domain(z=f32("dem", 0.0), mask=np.fromfile(d / "mask.bin", np.uint8, nr * nc).reshape(nr, nc),
                  n=f32("n", 0.03), C=f32("C", 0.0), Rday=f32("Rday", 0.0), h=h, dx=dx)


def read_field(path, name: str, shape) -> np.ndarray:
    """An output raster (hmax, h_final) the reference writes with
    fca_grid_write_field (float32, or float64 when its JSON says so)."""
    import json
    from pathlib import Path
    d = Path(path)
    dt = np.float32
    j = d / f"{name}.json"
    if j.exists() and json.loads(j.read_text()).get("dtype") == "float64":
        dt = np.float64
    return np.fromfile(d / f"{name}.bin", dt).reshape(shape)


def write_field(path, name: str, arr: np.ndarray, dx: float, x0: float = 0.0,
                y0: float = 0.0) -> None:
    """Writes an output raster (hmax, h_final, ...) as the reference's
    fca_grid_write_field does (src/common/grid.c:271-306): <name>.bin, raw
    float32 (float64 for a float64 array, the FCA_DOUBLE build), and a
    <name>.json header with the grid's shape, dx, dtype, CRS and origin."""
    import json
    import time
    from pathlib import Path
    d = Path(path)
    d.mkdir(parents=True, exist_ok=True)
    a = np.ascontiguousarray(arr, np.float64 if arr.dtype == np.float64 else np.float32)
    a.tofile(d / f"{name}.bin")
    nr, nc = a.shape
    hdr = {"name": name, "nrows": int(nr), "ncols": int(nc), "dx": float(np.float32(dx)),
           "dtype": "float64" if a.dtype == np.float64 else "float32", "crs": "EPSG:32643",
           "x0": float(x0), "y0": float(y0), "nodata": -9999, "source": "floodca",
           "created": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()), "sha256": ""}
    (d / f"{name}.json").write_text(json.dumps(hdr, separators=(",", ":")) + "\n")
