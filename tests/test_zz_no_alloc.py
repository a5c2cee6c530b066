"""fcab_run_noalloc: the allocation-free entry point gives the same depths as
the session entry point.

The entry point exists for callers that cannot call cudaMalloc (their device
memory belongs to another allocator, or they must not allocate while
running because allocation synchronises the device); it keeps its working
memory in a fixed library-global device array. The test calls it twice in a
row through the C-ABI, on two different grids, and compares each result with
the session path (fcab_sim_*), within the tolerance of the other GPU parity
tests. The arrays handed to it are allocated here, by the test.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import GOLDEN
from floodca_b200.abi import FcabStats
from floodca_b200.lib import core, last_error
from floodca_b200.sim import make_config, run_session
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
