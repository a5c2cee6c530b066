"""fcab_run_noalloc: the allocation-free entry point gives the same depths as
the session entry point and as the oracle.

The entry point exists for callers that cannot call cudaMalloc (their device
memory belongs to another allocator, or they must not allocate while
running because allocation synchronises the device); it keeps its working
memory in a fixed library-global device array. The tests call it twice in a
row through the C-ABI, on different grids, and compare each result with the
session path (fcab_sim_*) and with the CPU oracle (oracle/), within the
tolerance of the other GPU parity tests. The arrays handed to it are
allocated here, by the test.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import GOLDEN
from floodca_b200.abi import FcabStats
from floodca_b200.lib import core, last_error
from floodca_b200.sim import make_config, run_session
from oracle import pyoracle
from tests.golden.make_golden import load_case

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _noalloc(dom, p):
    import torch
    d = dom.astype(np.float32)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    z, n, Cc, R, m = dev(d.z), dev(d.n), dev(d.C), dev(d.Rday), dev(d.mask)
    h, hmax = dev(d.h), dev(d.h)
    tmax = torch.zeros_like(h)
    cfg = make_config(d, p, precision="f32")
    st = FcabStats()
    ptr = lambda t: C.c_void_p(t.data_ptr())
    torch.cuda.synchronize()
    rc = core().fcab_run_noalloc(C.byref(cfg), ptr(z), ptr(n), ptr(Cc), ptr(R), ptr(m), ptr(h),
                                 ptr(hmax), ptr(tmax), None, C.byref(st))
    assert rc == 0, last_error()
    torch.cuda.synchronize()
    return {"h": h.cpu().numpy(), "hmax": hmax.cpu().numpy(), "tmax": tmax.cpu().numpy(),
            **st.as_dict()}


def _enqueue_noalloc(dom, p, stream):
    """Enqueues one call on `stream` (a torch.cuda.Stream) with tmax and stats
    NULL; returns the device arrays (kept alive by the caller) and h, hmax."""
    import torch
    d = dom.astype(np.float32)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    arrs = [dev(d.z), dev(d.n), dev(d.C), dev(d.Rday), dev(d.mask), dev(d.h), dev(d.h)]
    torch.cuda.synchronize()
    z, n, Cc, R, m, h, hmax = arrs
    cfg = make_config(d, p, precision="f32")
    ptr = lambda t: C.c_void_p(t.data_ptr())
    rc = core().fcab_run_noalloc(C.byref(cfg), ptr(z), ptr(n), ptr(Cc), ptr(R), ptr(m), ptr(h),
                                 ptr(hmax), None, C.c_void_p(stream.cuda_stream), None)
    assert rc == 0, last_error()
    return arrs, h, hmax


def _case(name, steps):
    d, p, _, _ = load_case(GOLDEN / f"{name}.npz")
    return d, p.with_(steps=steps)


def test_noalloc_matches_session_on_two_calls():
    # a generic grid (SEA, WALL, spatial rain, all edges open) and an all-LAND
    # grid with box rain and an open south edge, one call after the other
    for name, steps in (("mixed_k4", 250), ("c1_64", 120)):
        d, p = _case(name, steps)
        want = run_session(d, p, precision="f32")
        got = _noalloc(d, p)
        assert got["step"] == want["step"] == steps
        for k in ("h", "hmax", "tmax"):
            diff = float(np.abs(got[k].astype(np.float64) - want[k]).max())
            assert diff <= (TOL if k != "tmax" else 1e-3), f"{name} {k}: {diff}"
        for k in ("V", "V_rain", "V_bnd", "V_sea"):
            assert got[k] == pytest.approx(want[k], rel=1e-9, abs=1e-6), f"{name} {k}"
        assert got["cap_total"] == want["cap_total"] > 0
        assert got["cap_active"] == want["cap_active"]


def test_noalloc_rejects_grid_beyond_capacity():
    import torch
    d, p = _case("tiny_3x3", 5)
    cfg = make_config(d, p, precision="f32")
    cfg.nrows, cfg.ncols = 2048, 2048
    x = torch.zeros(16, device="cuda")
    ptr = C.c_void_p(x.data_ptr())
    ptr2 = C.c_void_p(x.data_ptr() + 8)
    rc = core().fcab_run_noalloc(C.byref(cfg), ptr, ptr, None, None, ptr, ptr, ptr2, None, None,
                                 None)
    assert rc != 0 and "limit" in last_error()


def _inflow_on_land(d, p):
    land = np.flatnonzero(d.mask.ravel() == 0)
    cell = int(land[len(land) // 3])
    return p.with_(inflow_cell=cell, inflow_peak=40.0, inflow_t_peak=1200.0, inflow_t_end=4000.0)


def test_noalloc_on_a_stream_matches_oracle_back_to_back():
    # a K = 8, U = 3 grid with SEA/WALL cells, a rain field and an inflow
    # cell, then an all-LAND grid with box rain and an open south edge;
    # tmax and stats NULL, both calls enqueued on one stream with no host
    # wait between them
    import torch
    d1, p1 = _case("mixed_k8", 300)
    p1 = _inflow_on_land(d1, p1)
    d2, p2 = _case("inflow", 150)
    stream = torch.cuda.Stream()
    keep1, h1, hm1 = _enqueue_noalloc(d1, p1, stream)
    keep2, h2, hm2 = _enqueue_noalloc(d2, p2, stream)
    stream.synchronize()
    for d, p, h, hm in ((d1, p1, h1, hm1), (d2, p2, h2, hm2)):
        want = run_session(d, p, precision="f32")
        ref = pyoracle.run(d, p)
        assert want["step"] == ref["step"] == p.steps
        got = {"h": h.cpu().numpy(), "hmax": hm.cpu().numpy()}
        for k in ("h", "hmax"):
            for other in (want, ref):
                diff = float(np.abs(got[k].astype(np.float64) - other[k]).max())
                assert diff <= TOL, f"{k}: {diff}"


def test_noalloc_inflow_on_a_non_land_cell_adds_nothing():
    d, p = _case("mixed_k4", 80)
    sea = int(np.flatnonzero(d.mask.ravel() == 1)[0])
    got = _noalloc(d, p.with_(inflow_cell=sea, inflow_peak=40.0, inflow_t_peak=600.0,
                              inflow_t_end=3000.0))
    base = _noalloc(d, p)
    assert got["V_in"] == 0.0
    assert np.array_equal(got["h"], base["h"]) and np.array_equal(got["hmax"], base["hmax"])
    assert got["cap_total"] == base["cap_total"] > 0
