"""ctypes front end of the C oracle (oracle/wca_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path. Only tests/,
__graft_entry__.smoke() and bench.py's cpu_baseline leg import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from functools import lru_cache
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


class OrParams(C.Structure):
    _fields_ = [
        ("dx", C.c_double), ("g", C.c_double), ("alpha", C.c_double), ("tau_h", C.c_double),
        ("tau_l", C.c_double), ("z_sea", C.c_double), ("dt_max", C.c_double),
        ("dt_min", C.c_double), ("S_bnd", C.c_double),
        ("U", C.c_int), ("K", C.c_int), ("boundary", C.c_int),
        ("edge_n", C.c_int), ("edge_s", C.c_int), ("edge_w", C.c_int), ("edge_e", C.c_int),
        ("T_sim", C.c_double), ("out_every", C.c_double), ("hyeto", C.c_int),
        ("D_h", C.c_double), ("phi", C.c_double), ("lambda_", C.c_double),
        ("rain_end", C.c_double), ("inflow_cell", C.c_longlong),
        ("inflow_peak", C.c_double), ("inflow_t_peak", C.c_double), ("inflow_t_end", C.c_double),
        ("steps", C.c_int), ("n_force_days", C.c_int),
    ]


class OrAcc(C.Structure):
    _fields_ = [
        ("V", C.c_double), ("V0", C.c_double), ("V_rain", C.c_double), ("V_sea", C.c_double),
        ("V_bnd", C.c_double), ("clamp_err", C.c_double), ("V_in", C.c_double),
        ("cap_active", C.c_longlong), ("cap_total", C.c_longlong), ("dt_min_hits", C.c_longlong),
        ("t", C.c_double), ("step", C.c_int), ("dt_base", C.c_double), ("force_day", C.c_int),
    ]


def ensure_built() -> None:
    libs = [HERE / "liboracle_f32.so", HERE / "liboracle_f64.so"]
    srcs = [HERE / "wca_oracle.c", HERE / "wca_oracle.h"]
    if all(l.exists() for l in libs) and all(
            l.stat().st_mtime >= max(s.stat().st_mtime for s in srcs) for l in libs):
        return
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


@lru_cache(maxsize=2)
def lib(double: bool) -> C.CDLL:
    ensure_built()
    L = C.CDLL(str(HERE / ("liboracle_f64.so" if double else "liboracle_f32.so")))
    vp = C.c_void_p
    L.or_run.restype = C.c_int
    L.or_run.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, C.POINTER(OrParams),
                         C.POINTER(OrAcc), C.c_int, vp]
    L.or_acc_init.restype = None
    L.or_acc_init.argtypes = [C.POINTER(OrAcc), C.c_int, C.c_int, vp, vp, C.c_double]
    L.or_mass_error.restype = C.c_double
    L.or_mass_error.argtypes = [C.POINTER(OrAcc)]
    L.or_hyeto_integral.restype = C.c_double
    L.or_hyeto_integral.argtypes = [C.POINTER(OrParams), C.c_double, C.c_double]
    L.or_next_event_time.restype = C.c_double
    L.or_next_event_time.argtypes = [C.POINTER(OrParams), C.c_double]
    L.or_inflow_volume.restype = C.c_double
    L.or_inflow_volume.argtypes = [C.POINTER(OrParams), C.c_double, C.c_double]
    real = C.c_double if double else C.c_float
    L.or_cbrt_sq.restype = real
    L.or_cbrt_sq.argtypes = [real]
    L.or_real_size.restype = C.c_int
    return L


def params_of(dom, p) -> OrParams:
    q = OrParams()
    q.dx, q.g, q.alpha, q.tau_h, q.tau_l = dom.dx, p.g, p.alpha, p.tau_h, p.tau_l
    q.z_sea, q.dt_max, q.dt_min, q.S_bnd = p.z_sea, p.dt_max, p.dt_min, p.S_bnd
    q.U, q.K = p.U, p.K
    q.boundary = 0 if p.boundary == "open" else 1
    q.edge_n, q.edge_s, q.edge_w, q.edge_e = p.edges
    q.T_sim, q.out_every = p.T_sim, p.out_every
    q.hyeto = 1 if p.hyeto == "uniform" else 0
    q.D_h, q.phi, q.lambda_ = p.D_h, p.phi, p.lambda_
    q.rain_end = p.rain_end
    q.inflow_cell = p.inflow_cell
    q.inflow_peak, q.inflow_t_peak, q.inflow_t_end = p.inflow_peak, p.inflow_t_peak, p.inflow_t_end
    q.steps = p.steps
    q.n_force_days = 0
    return q


def run(dom, p, double: bool = False, max_calls: int = 2_000_000_000, threads: int | None = None,
        force_rday: np.ndarray | None = None) -> dict:
    """Runs the oracle on a copy of the domain; returns h, hmax, tmax and the
    accumulators (FloodCA fca_run semantics plus the extensions)."""
    if threads:
        os.environ["OMP_NUM_THREADS"] = str(threads)
    dt = np.float64 if double else np.float32
    cp = lambda a: np.ascontiguousarray(a, dtype=dt).copy()
    z, n, Cc = cp(dom.z), cp(dom.n), cp(dom.C)
    R = cp(dom.Rday)
    if dt(p.lambda_) != dt(1) and force_rday is None:
        R = (R * dt(p.lambda_)).astype(dt)
    h = cp(dom.h)
    hmax = cp(dom.hmax if dom.hmax is not None else dom.h)
    tmax = cp(dom.tmax) if dom.tmax is not None else np.zeros_like(h)
    mask = np.ascontiguousarray(dom.mask, np.uint8)
    nr, nc = h.shape
    q = params_of(dom, p)
    fr = None
    if force_rday is not None:
        fr = np.ascontiguousarray(force_rday, dtype=dt)
        q.n_force_days = fr.shape[0]
    L = lib(double)
    acc = OrAcc()
    vp = lambda a: a.ctypes.data_as(C.c_void_p)
    L.or_acc_init(C.byref(acc), nr, nc, vp(h), vp(mask), dom.dx)
    taken = L.or_run(nr, nc, vp(z), vp(h), vp(n), vp(Cc), vp(R), vp(mask), vp(hmax), vp(tmax),
                     C.byref(q), C.byref(acc), max_calls, None if fr is None else vp(fr))
    if taken < 0:
        raise RuntimeError("oracle run failed")
    out = {f[0]: getattr(acc, f[0]) for f in acc._fields_}
    out["E_mass"] = L.or_mass_error(C.byref(acc))
    out.update(h=h, hmax=hmax, tmax=tmax, taken=taken)
    return out
