"""Python host layer over the fcab_* sessions and the drop-in fca_cuda_* ABI.

Domain holds the row-major rasters the reference reads from a grid
directory (FloodCA src/common/grid.c:162-237); RunParams holds FloodCA's
run parameters (src/common/config.c:8-131) plus the extensions this project
adds (per-edge open boundary, rain end time, point inflow).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field, replace

import numpy as np

from . import abi
from .abi import FcabConfig, FcabInfo, FcabPoll, FcabStats
from .lib import check, core, dropin

PREC = {"f32": abi.FCAB_PREC_F32, "f32all": abi.FCAB_PREC_F32_ALL, "f64": abi.FCAB_PREC_F64}
MATH = {"exact": abi.FCAB_MATH_EXACT, "fast": abi.FCAB_MATH_FAST}


@dataclass
class Domain:
    """Row-major rasters of one grid. Arrays are float32 (or float64 for the
    f64 precision) except mask (uint8: 0 LAND, 1 SEA, 2 WALL)."""
    z: np.ndarray
    mask: np.ndarray
    n: np.ndarray
    C: np.ndarray
    Rday: np.ndarray
    h: np.ndarray
    dx: float
    hmax: np.ndarray | None = None
    tmax: np.ndarray | None = None

    @property
    def shape(self) -> tuple[int, int]:
        return self.z.shape

    def astype(self, dtype) -> "Domain":
        cv = lambda a: None if a is None else np.ascontiguousarray(a, dtype=dtype)
        return Domain(cv(self.z), np.ascontiguousarray(self.mask, np.uint8), cv(self.n),
                      cv(self.C), cv(self.Rday), cv(self.h), self.dx, cv(self.hmax),
                      cv(self.tmax))

    def copy(self) -> "Domain":
        cp = lambda a: None if a is None else a.copy()
        return Domain(cp(self.z), cp(self.mask), cp(self.n), cp(self.C), cp(self.Rday),
                      cp(self.h), self.dx, cp(self.hmax), cp(self.tmax))


@dataclass
class RunParams:
    """Reference defaults (FloodCA src/common/config.c:8-45) and extensions."""
    K: int = 4
    U: int = 1
    boundary: str = "open"                      # "open" | "closed"
    edges: tuple = (1, 1, 1, 1)                 # open edges (n, s, w, e)
    hyeto: str = "triangle"                     # "triangle" | "uniform"
    D_h: float = 24.0
    phi: float = 0.5
    lambda_: float = 1.0
    T_sim: float = 86400.0
    out_every: float = 0.0
    steps: int = 0
    g: float = 9.81
    alpha: float = 0.5
    tau_h: float = 1e-3
    tau_l: float = 1e-5
    z_sea: float = 0.0
    dt_max: float = 60.0
    dt_min: float = 0.01
    S_bnd: float = 0.001
    rain_end: float = 0.0                       # extension: rain stops at this time
    inflow_cell: int = -1                       # extension: point hydrograph cell
    inflow_peak: float = 0.0
    inflow_t_peak: float = 0.0
    inflow_t_end: float = 0.0

    def with_(self, **kw) -> "RunParams":
        return replace(self, **kw)


def make_config(dom, p: RunParams, precision="f32", math="exact", cols_per_lane=0,
                seg_rows=0) -> FcabConfig:
    """dom: a Domain, or anything with .shape (rows, cols) and .dx."""
    c = FcabConfig()
    core().fcab_config_defaults(C.byref(c), dom.shape[0], dom.shape[1])
    c.precision, c.math = PREC[precision], MATH[math]
    c.K, c.U = p.K, p.U
    c.boundary = abi.FCA_BND_OPEN if p.boundary == "open" else abi.FCA_BND_CLOSED
    c.edge_n, c.edge_s, c.edge_w, c.edge_e = p.edges
    c.hyeto = abi.FCA_HYETO_UNIFORM if p.hyeto == "uniform" else abi.FCA_HYETO_TRIANGLE
    c.max_steps = p.steps
    c.dx, c.g, c.alpha, c.tau_h, c.tau_l = dom.dx, p.g, p.alpha, p.tau_h, p.tau_l
    c.z_sea, c.dt_max, c.dt_min, c.S_bnd = p.z_sea, p.dt_max, p.dt_min, p.S_bnd
    c.T_sim, c.out_every, c.D_h, c.phi = p.T_sim, p.out_every, p.D_h, p.phi
    c.rain_end = p.rain_end
    c.inflow_cell = p.inflow_cell
    c.inflow_peak, c.inflow_t_peak, c.inflow_t_end = p.inflow_peak, p.inflow_t_peak, p.inflow_t_end
    c.cols_per_lane, c.seg_rows = cols_per_lane, seg_rows
    return c


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def effective_rday(dom: Domain, p: RunParams, dtype) -> np.ndarray:
    """Rday as the reference applies lambda to a rain field (grid.c:256-268)."""
    R = np.ascontiguousarray(dom.Rday, dtype=dtype)
    if dtype(p.lambda_) != dtype(1):
        R = (R * dtype(p.lambda_)).astype(dtype)
    return R


class Session:
    """A device-resident run of one domain on the current GPU."""

    def __init__(self, dom: Domain, p: RunParams, precision: str = "f32", math: str = "exact",
                 cols_per_lane: int = 0, seg_rows: int = 0, stream=None):
        self.dom = dom.astype(np.float64 if precision == "f64" else np.float32)
        self._create(self.dom, p, precision, math, cols_per_lane, seg_rows, stream)
        d = self.dom
        R = effective_rday(d, p, self.dtype)
        check(self.L.fcab_sim_upload(self.h, _ptr(d.z), _ptr(d.h), _ptr(d.n), _ptr(d.C), _ptr(R),
                                     _ptr(d.mask), _ptr(d.hmax), _ptr(d.tmax)), "fcab_sim_upload")

    def _create(self, dom, p, precision, math, cols_per_lane, seg_rows, stream):
        self.L = core()
        self.precision = precision
        self.dtype = np.float64 if precision == "f64" else np.float32
        self.shape = tuple(dom.shape)
        self.p = p
        self.cfg = make_config(dom, p, precision, math, cols_per_lane, seg_rows)
        h = C.c_void_p()
        check(self.L.fcab_sim_create(C.byref(h), C.byref(self.cfg), stream), "fcab_sim_create")
        self.h = h

    @classmethod
    def from_device(cls, shape, dx: float, p: RunParams, z, h, mask, n=None, Cf=None,
                    Rday=None, precision: str = "f32", math: str = "exact",
                    cols_per_lane: int = 0, seg_rows: int = 0, stream=None) -> "Session":
        """A session uploaded from device arrays (row-major, contiguous, of the
        precision's element type; mask uint8), given as raw pointers or as
        objects with data_ptr(). Rday is used as given (lambda already applied)."""
        from types import SimpleNamespace
        s = cls.__new__(cls)
        s.dom = None
        s._create(SimpleNamespace(shape=tuple(shape), dx=dx), p, precision, math,
                  cols_per_lane, seg_rows, stream)
        ptr = lambda a: None if a is None else C.c_void_p(a.data_ptr() if hasattr(a, "data_ptr")
                                                           else int(a))
        check(s.L.fcab_sim_upload_device(s.h, ptr(z), ptr(h), ptr(n), ptr(Cf), ptr(Rday),
                                         ptr(mask), None, None), "fcab_sim_upload_device")
        return s

    # -- running -------------------------------------------------------------
    def advance(self, nsteps: int) -> None:
        check(self.L.fcab_sim_advance(self.h, int(nsteps)), "fcab_sim_advance")

    def run(self) -> "Session":
        check(self.L.fcab_sim_run(self.h), "fcab_sim_run")
        return self

    def poll(self) -> FcabPoll:
        p = FcabPoll()
        check(self.L.fcab_sim_poll(self.h, C.byref(p)), "fcab_sim_poll")
        return p

    def stats(self) -> dict:
        st = FcabStats()
        check(self.L.fcab_sim_stats(self.h, C.byref(st)), "fcab_sim_stats")
        return st.as_dict()

    def info(self) -> dict:
        i = FcabInfo()
        check(self.L.fcab_sim_info(self.h, C.byref(i)), "fcab_sim_info")
        return {f[0]: getattr(i, f[0]) for f in i._fields_}

    def download(self):
        nr, nc = self.shape
        h = np.empty((nr, nc), self.dtype)
        hmax = np.empty((nr, nc), self.dtype)
        tmax = np.empty((nr, nc), self.dtype)
        check(self.L.fcab_sim_download(self.h, _ptr(h), _ptr(hmax), _ptr(tmax)),
              "fcab_sim_download")
        return h, hmax, tmax

    def count_flooded(self, thresholds=(0.10, 0.25, 0.50), counts=None):
        """LAND cells with hmax >= each threshold and the largest LAND hmax;
        counts: optional device uint16 raster [len(thresholds), rows, cols]
        (a torch tensor) that the flooded cells are added into."""
        n = len(thresholds)
        thr = (C.c_double * n)(*thresholds)
        fl = (C.c_longlong * n)()
        mx = C.c_double()
        cp = None if counts is None else C.c_void_p(counts.data_ptr())
        check(self.L.fcab_sim_count_flooded(self.h, n, thr, cp, fl, C.byref(mx)),
              "fcab_sim_count_flooded")
        return [int(v) for v in fl], float(mx.value)

    def write_outputs(self, out_dir) -> None:
        """hmax and h_final in the reference's output format, as its CLIs
        write them (src/cuda/main_cuda.c:73-80)."""
        from .synth import write_field
        h, hmax, _ = self.download()
        write_field(out_dir, "hmax", hmax, self.cfg.dx)
        write_field(out_dir, "h_final", h, self.cfg.dx)

    def launches(self) -> int:
        return int(self.L.fcab_sim_launches(self.h))

    def stream(self):
        return self.L.fcab_sim_stream(self.h)

    def close(self) -> None:
        if getattr(self, "h", None):
            self.L.fcab_sim_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def run_session(dom: Domain, p: RunParams, **kw) -> dict:
    """Runs to the end and returns h, hmax, tmax and the stats."""
    with Session(dom, p, **kw) as s:
        s.run()
        st = s.stats()
        h, hmax, tmax = s.download()
    return {"h": h, "hmax": hmax, "tmax": tmax, **st}


# ---------------------------------------------------------------------------
# The reference-facing C-ABI (fca_cuda_run), called with host buffers.

class DropinGrid:
    """Builds FcaGrid/FcaRunCfg/FcaAcc/FcaTimers for fca_cuda_run from a
    Domain, with the host arrays owned by this object."""

    def __init__(self, dom: Domain, p: RunParams, double: bool = False):
        self.double = double
        self.T = abi.fca_types(C.c_double if double else C.c_float)
        dt = np.float64 if double else np.float32
        d = dom.astype(dt)
        nr, nc = d.shape
        self.arrays = {
            "z": d.z, "h": d.h.copy(), "n": d.n, "C": d.C,
            "Rday": effective_rday(d, p, dt).copy(), "mask": d.mask,
            "hmax": (d.hmax if d.hmax is not None else d.h).copy(),
            "tmax": (d.tmax if d.tmax is not None else np.zeros_like(d.h)).copy(),
        }
        T = self.T
        g = T.FcaGrid()
        g.nrows, g.ncols = nr, nc
        g.r0, g.r1, g.c0, g.c1 = 0, nr, 0, nc
        g.edge_n, g.edge_s, g.edge_w, g.edge_e = p.edges
        g.dx = dom.dx
        rp = C.POINTER(T.real)
        for k in ("z", "h", "n", "C", "Rday", "hmax", "tmax"):
            setattr(g, k, self.arrays[k].ctypes.data_as(rp))
        g.mask = self.arrays["mask"].ctypes.data_as(C.POINTER(C.c_uint8))
        self.g = g
        cfg = T.FcaRunCfg()
        ph = cfg.phys
        ph.dx = dom.dx
        ph.A = T.real(dom.dx).value * T.real(dom.dx).value
        ph.A = float(np.array(dom.dx, dt) * np.array(dom.dx, dt))
        ph.g, ph.alpha, ph.tau_h, ph.tau_l = p.g, p.alpha, p.tau_h, p.tau_l
        ph.z_sea, ph.dt_max, ph.dt_min, ph.S_bnd, ph.h_flood = p.z_sea, p.dt_max, p.dt_min, p.S_bnd, 0.25
        ph.U, ph.K = p.U, p.K
        ph.boundary = abi.FCA_BND_OPEN if p.boundary == "open" else abi.FCA_BND_CLOSED
        cfg.T_sim, cfg.out_every = p.T_sim, p.out_every
        cfg.hyeto = abi.FCA_HYETO_UNIFORM if p.hyeto == "uniform" else abi.FCA_HYETO_TRIANGLE
        cfg.D_h, cfg.phi, cfg.lambda_ = p.D_h, p.phi, p.lambda_
        cfg.steps, cfg.neigh = p.steps, p.K
        cfg.block_x = cfg.block_y = 16
        cfg.diag_every = 100
        self.cfg = cfg
        acc = T.FcaAcc()
        A = float(np.array(dom.dx, dt) * np.array(dom.dx, dt))
        land = d.mask == abi.FCA_LAND
        acc.V0 = float(np.sum(d.h[land].astype(np.float64) * A))
        acc.V = acc.V0
        acc.force_day = -1
        self.acc = acc
        tm = T.FcaTimers()
        tm.t_h2d = tm.t_d2h = tm.t_halo = tm.t_allreduce = tm.bytes_per_step = -1
        self.tm = tm

    def run(self) -> int:
        L = dropin(self.double)
        return L.fca_cuda_run(C.byref(self.g), C.byref(self.cfg), C.byref(self.acc),
                              C.byref(self.tm))

    def result(self) -> dict:
        a = self.acc
        out = {k: getattr(a, k) for k, _ in a._fields_}
        out.update(h=self.arrays["h"], hmax=self.arrays["hmax"], tmax=self.arrays["tmax"])
        return out
