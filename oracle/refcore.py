"""Harness around the FloodCA reference core compiled in oracle/_ref/.

TEST INFRASTRUCTURE ONLY. oracle/Makefile.ref compiles the reference's own
src/common/*.c (unmodified, read in place) into libfcaref_*.so; this module
calls its public functions (fca_acc_init, fca_step, fca_run,
fca_next_event_time from src/common/model.h and rain.h) through ctypes with
the ABI structs of floodca_b200.abi.

It produces the golden fixtures (tests/golden/make_golden.py) and is the
`reference` CPU baseline of bench.py. The reference CLI cannot express three
features of the benchmark workloads; the harness adds them around fca_step
without touching the physics:
  * per-edge open boundary: the FcaGrid edge_n/s/w/e flags, which fca_step
    already honours (src/common/model.c:130-132, 453-476);
  * rain that stops at rain_end: out_every must make a step land on
    rain_end; Rday is zeroed once t >= rain_end;
  * a point inflow: after each step, V_in (exact integral of the triangular
    hydrograph over the step) is added to the inflow cell as V_in/A, then
    hmax/tmax are updated, which equals doing it after the clamp and before
    the hmax test inside the step.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from functools import lru_cache
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
ROOT = HERE.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from floodca_b200 import abi  # noqa: E402


def available(kind: str = "f32") -> bool:
    return (REF_DIR / f"libfcaref_{kind}.so").exists()


def build(ref_root: str = "/root/reference") -> bool:
    """Compiles the reference core into oracle/_ref when its sources exist."""
    if not Path(ref_root, "src/common/model.c").exists():
        return False
    subprocess.run(["make", "-s", "-f", str(HERE / "Makefile.ref"), f"REF={ref_root}", "-j4"],
                   check=True)
    # the reference's CUDA CLI linked against the drop-in library, once it is built
    if (ROOT / "floodca_b200" / "libfloodca_b200.so").exists():
        subprocess.run(["make", "-s", "-f", str(HERE / "Makefile.ref"), f"REF={ref_root}",
                        "dropin"], check=True)
    # the same CLI on the reference's own CUDA backend (same-box GPU comparison)
    subprocess.run(["make", "-s", "-f", str(HERE / "Makefile.ref"), f"REF={ref_root}",
                    "refcuda"], check=True)
    return True


def shipped_kind() -> str:
    """The release-flag build this host can run: AVX-512 (v4) or AVX2 (v3)."""
    try:
        flags = Path("/proc/cpuinfo").read_text()
    except OSError:
        flags = ""
    return "shipped_v4" if " avx512f" in flags and " avx512bw" in flags else "shipped_v3"


@lru_cache(maxsize=4)
def lib(kind: str = "f32") -> C.CDLL:
    path = REF_DIR / f"libfcaref_{kind}.so"
    if not path.exists():
        raise FileNotFoundError(f"{path} missing: build with `make -f oracle/Makefile.ref`")
    L = C.CDLL(str(path))
    double = kind == "f64"
    T = abi.fca_types(C.c_double if double else C.c_float)
    L.fca_acc_init.restype = None
    L.fca_acc_init.argtypes = [C.POINTER(T.FcaAcc), C.POINTER(T.FcaGrid), T.real]
    L.fca_step.restype = None
    L.fca_step.argtypes = [C.POINTER(T.FcaGrid), C.POINTER(T.FcaRunCfg), C.POINTER(T.FcaAcc),
                           C.POINTER(T.FcaTimers), C.c_double]
    L.fca_run.restype = C.c_int
    L.fca_run.argtypes = [C.POINTER(T.FcaGrid), C.POINTER(T.FcaRunCfg), C.POINTER(T.FcaAcc),
                          C.POINTER(T.FcaTimers)]
    L.fca_next_event_time.restype = C.c_double
    L.fca_next_event_time.argtypes = [C.POINTER(T.FcaRunCfg), C.c_double]
    L.fca_volume_land.restype = C.c_double
    L.fca_volume_land.argtypes = [C.POINTER(T.FcaGrid), T.real]
    L.fca_mass_error.restype = C.c_double
    L.fca_mass_error.argtypes = [C.POINTER(T.FcaAcc)]
    L.fca_timers_init.restype = None
    L.fca_timers_init.argtypes = [C.POINTER(T.FcaTimers)]
    L.fca_cfg_defaults.restype = None
    L.fca_cfg_defaults.argtypes = [C.POINTER(T.FcaRunCfg)]
    L.T = T
    L.double = double
    return L


def inflow_volume(p, t: float, dt: float) -> float:
    """Exact integral of the triangular hydrograph (0 at t=0, peak at
    inflow_t_peak, 0 at inflow_t_end) over [t, t+dt]; same rule as the oracle."""
    if p.inflow_cell < 0 or dt <= 0.0:
        return 0.0
    tp, te, Qp = p.inflow_t_peak, p.inflow_t_end, p.inflow_peak

    def q(x):
        if x <= 0.0 or x >= te:
            return 0.0
        if x <= tp:
            return Qp * (x / tp) if tp > 0.0 else Qp
        return Qp * ((te - x) / (te - tp)) if te > tp else 0.0

    t1 = t + dt
    t = max(t, 0.0)
    t1 = min(t1, te)
    a, s = t, 0.0
    while a < t1:
        b = tp if (a < tp and t1 > tp) else t1
        s += 0.5 * (q(a) + q(b)) * (b - a)
        a = b
    return s


class RefRun:
    """One reference run on a Domain (floodca_b200.sim.Domain)."""

    def __init__(self, dom, p, kind: str = "f32", force_files: list[str] | None = None):
        self.L = lib(kind)
        T = self.L.T
        self.p = p
        dt = np.float64 if self.L.double else np.float32
        self.dt = dt
        d = dom.astype(dt)
        nr, nc = d.shape
        N = nr * nc
        self.keep = {
            "z": d.z.copy(), "h": d.h.copy(), "n": d.n.copy(), "C": d.C.copy(),
            "Rday": d.Rday.copy(), "mask": d.mask.copy(),
            "hmax": (d.hmax if d.hmax is not None else d.h).copy(),
            "tmax": (d.tmax if d.tmax is not None else np.zeros_like(d.h)).copy(),
            "s": np.ones(N, dt), "out": np.zeros(N, dt),
            "Qx": np.zeros(max(1, nr * (nc - 1)), dt), "Qy": np.zeros(max(1, (nr - 1) * nc), dt),
            "Qd1": np.zeros(max(1, (nr - 1) * (nc - 1)), dt),
            "Qd2": np.zeros(max(1, (nr - 1) * (nc - 1)), dt), "Qopen": np.zeros(4 * N, dt),
        }
        if dt(p.lambda_) != dt(1) and not force_files:
            self.keep["Rday"] = (self.keep["Rday"] * dt(p.lambda_)).astype(dt)
        g = T.FcaGrid()
        g.nrows, g.ncols = nr, nc
        g.r0, g.r1, g.c0, g.c1 = 0, nr, 0, nc
        g.edge_n, g.edge_s, g.edge_w, g.edge_e = p.edges
        g.dx = dom.dx
        rp = C.POINTER(T.real)
        for k, a in self.keep.items():
            if k == "mask":
                g.mask = a.ctypes.data_as(C.POINTER(C.c_uint8))
            else:
                setattr(g, k, a.ctypes.data_as(rp))
        self.g = g
        cfg = T.FcaRunCfg()
        self.L.fca_cfg_defaults(C.byref(cfg))
        ph = cfg.phys
        ph.dx = dom.dx
        ph.A = float(np.array(dom.dx, dt) * np.array(dom.dx, dt))
        ph.g, ph.alpha, ph.tau_h, ph.tau_l = p.g, p.alpha, p.tau_h, p.tau_l
        ph.z_sea, ph.dt_max, ph.dt_min, ph.S_bnd = p.z_sea, p.dt_max, p.dt_min, p.S_bnd
        ph.U, ph.K = p.U, p.K
        ph.boundary = abi.FCA_BND_OPEN if p.boundary == "open" else abi.FCA_BND_CLOSED
        cfg.neigh = p.K
        cfg.T_sim, cfg.out_every = p.T_sim, p.out_every
        cfg.hyeto = abi.FCA_HYETO_UNIFORM if p.hyeto == "uniform" else abi.FCA_HYETO_TRIANGLE
        cfg.D_h, cfg.phi, cfg.lambda_ = p.D_h, p.phi, p.lambda_
        cfg.steps = p.steps
        cfg.progress_every = 0
        if force_files:
            cfg.n_force_days = len(force_files)
            for i, f in enumerate(force_files):
                cfg.force_files[i].value = f.encode()
        self.cfg = cfg
        self.acc = T.FcaAcc()
        self.L.fca_acc_init(C.byref(self.acc), C.byref(g), ph.A)
        self.tm = T.FcaTimers()
        self.L.fca_timers_init(C.byref(self.tm))
        self.V_in = 0.0
        self.inflow_ok = 0 <= p.inflow_cell < N and self.keep["mask"].ravel()[p.inflow_cell] == 0

    @property
    def plain(self) -> bool:
        return self.p.rain_end <= 0 and not self.inflow_ok

    def step(self) -> bool:
        """One reference step plus the harness extensions; False if it did not advance."""
        acc, p, dt = self.acc, self.p, self.dt
        t0, st = acc.t, acc.step
        if p.rain_end > 0 and not (p.rain_end - t0 >= 1e-9):
            self.keep["Rday"][...] = 0
        self.L.fca_step(C.byref(self.g), C.byref(self.cfg), C.byref(acc), C.byref(self.tm), 0.0)
        if acc.step == st:
            return False          # dt <= 0 or a forcing-file failure: no step taken
        if self.inflow_ok:
            # the step's dt, as fca_step derives it (src/common/model.c:366-378)
            dtr = dt(acc.dt_base)
            remain = self.L.fca_next_event_time(C.byref(self.cfg), t0) - t0
            if remain <= float(dtr):
                dtr = dt(max(remain, 0.0))
            V = inflow_volume(p, t0, float(dtr))
            a = p.inflow_cell
            A = float(dt(self.cfg.phys.A))
            h = self.keep["h"].reshape(-1)
            h[a] = dt(h[a] + dt(V / A))
            hm = self.keep["hmax"].reshape(-1)
            if h[a] > hm[a]:
                hm[a] = h[a]
                self.keep["tmax"].reshape(-1)[a] = dt(t0 + float(dtr))
            self.V_in += V
        return True

    def run(self, max_steps: int | None = None) -> "RefRun":
        acc, cfg, p = self.acc, self.cfg, self.p
        if self.plain and max_steps is None:
            self.L.fca_run(C.byref(self.g), C.byref(cfg), C.byref(acc), C.byref(self.tm))
            return self
        limit = p.steps if p.steps > 0 else 2_000_000_000
        taken = 0
        while acc.step < limit and (max_steps is None or taken < max_steps):
            if p.steps <= 0 and acc.t >= float(self.dt(p.T_sim)) - 1e-15:
                break
            if not self.step():
                break
            taken += 1
        acc.V = self.L.fca_volume_land(C.byref(self.g), cfg.phys.A)
        return self

    def result(self) -> dict:
        a = self.acc
        out = {f[0]: getattr(a, f[0]) for f in a._fields_}
        out["V_in"] = self.V_in
        den = max(a.V_rain + self.V_in + a.V0, 1e-30)
        out["E_mass"] = abs(a.V + a.V_sea + a.V_bnd - a.V_rain - self.V_in - a.V0 - a.clamp_err) / den
        out.update(h=self.keep["h"].copy(), hmax=self.keep["hmax"].copy(),
                   tmax=self.keep["tmax"].copy())
        return out


def run(dom, p, kind: str = "f32", threads: int | None = None, **kw) -> dict:
    if threads:
        os.environ["OMP_NUM_THREADS"] = str(threads)
    return RefRun(dom, p, kind, **kw).run().result()
