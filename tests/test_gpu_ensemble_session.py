"""The reference-facing ensemble session (fca_cuda_ens_*, FloodCA
src/cuda/kernels.cu:790-1043): each scenario run equals a plain run of the
same scenario and the compiled reference core's run of it (steps, time,
volumes), and the flooded-cell counts, the maximum depth and the uint16
count rasters are those of the reference core's hmax (hmax >= thr on LAND
cells, as k_ens_count does, src/cuda/kernels.cu:799-823)."""
import ctypes as C

import numpy as np
import pytest

from conftest import GOLDEN
from floodca_b200 import abi
from floodca_b200.lib import dropin
from floodca_b200.sim import DropinGrid
from tests import refpin
from tests.golden.make_golden import load_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("double", [False, True])
def test_ensemble_session_matches_single_runs(double):
    d, p, f, _ = load_case(GOLDEN / "mixed_k4.npz")
    L = dropin(double)
    thr = (C.c_double * 3)(0.10, 0.25, 0.50)
    base = DropinGrid(d, p, double=double)
    e = L.fca_cuda_ens_open(C.byref(base.g), C.byref(base.cfg), 3, thr)
    assert e
    rng = np.random.default_rng(5)
    want_counts = np.zeros((3,) + d.shape, np.int64)
    try:
        for scen in range(3):
            ds = d.copy()
            ds.Rday = (d.Rday * rng.uniform(0.5, 3.0)).astype(np.float32)
            g = DropinGrid(ds, p, double=double)
            fl = (C.c_long * 3)()
            mx = C.c_double()
            rc = L.fca_cuda_ens_run(e, C.byref(g.g), C.byref(g.cfg), C.byref(g.acc),
                                    C.byref(g.tm), fl, C.byref(mx), None, None, 0)
            assert rc == 0
            single = DropinGrid(ds, p, double=double)
            assert single.run() == 0
            r = single.result()
            assert g.acc.step == r["step"] and g.acc.t == r["t"]
            assert g.acc.V == pytest.approx(r["V"], rel=1e-12)
            assert g.acc.V_rain == pytest.approx(r["V_rain"], rel=1e-12)
            kind = "f64" if double else "f32"
            ref = refpin.reference(ds, p, kind)
            refpin.check(r, ref, kind, volumes=("V", "V_rain", "V_sea", "V_bnd", "clamp_err"))
            assert g.acc.step == ref["step"]
            assert g.acc.V_rain == pytest.approx(ref["V_rain"], rel=1e-9)
            land = ds.mask == abi.FCA_LAND
            hm = np.asarray(ref["hmax"], np.float64)
            for j, t in enumerate((0.10, 0.25, 0.50)):
                hit = land & (hm >= t)
                assert fl[j] == int(hit.sum())
                want_counts[j] += hit
            assert mx.value == pytest.approx(max(0.0, float(hm[land].max())), rel=1e-12)
        counts = np.zeros(3 * d.shape[0] * d.shape[1], np.uint16)
        assert L.fca_cuda_ens_counts(e, counts.ctypes.data_as(C.POINTER(C.c_uint16))) == 0
        assert np.array_equal(counts.reshape(want_counts.shape), want_counts)
    finally:
        L.fca_cuda_ens_close(e)
