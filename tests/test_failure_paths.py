"""Failure paths that need no GPU: invalid configurations are rejected by
fcab_sim_create before any CUDA call, with FCAB_ERR_ARG and a message, and
fca_cuda_run returns nonzero for them (-1 for a bad block shape, as the
reference's src/cuda/kernels.cu:634-638 does; -2 when the session cannot be
created). The reference itself validates almost nothing here (its config
parser, src/common/config.c, takes values as given); these checks stop the
values for which the step would divide by zero or never advance the clock.

Failure paths on the device (non-finite host rasters, missing and short
forcing files, a bounded wait that runs out) are in
tests/test_gpu_failure_paths.py and tests/test_gpu_unet.py."""
import ctypes as C
import math

import pytest

from floodca_b200 import abi, lib
from floodca_b200.sim import DropinGrid
from tests.golden.make_golden import load_case
from conftest import GOLDEN


def _cfg(**kw):
    c = abi.FcabConfig()
    lib.core().fcab_config_defaults(C.byref(c), 8, 8)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


BAD = [
    ({"nrows": 0}, "empty"),
    ({"ncols": -3}, "empty"),
    ({"K": 6}, "only 4 or 8"),
    ({"precision": 7}, "precision"),
    ({"math": 3}, "math"),
    ({"U": 0}, "dt reuse"),
    ({"boundary": 2}, "boundary"),
    ({"hyeto": 5}, "hyetograph"),
    ({"dx": 0.0}, "dx, g and alpha"),
    ({"dx": math.nan}, "dx, g and alpha"),
    ({"g": -9.81}, "dx, g and alpha"),
    ({"alpha": math.inf}, "dx, g and alpha"),
    ({"dt_max": 0.0}, "dt_max and dt_min"),
    ({"dt_min": -1.0}, "dt_max and dt_min"),
    ({"dt_min": math.nan}, "dt_max and dt_min"),
    ({"tau_h": -1e-3}, "tau_h and tau_l"),
    ({"tau_l": math.nan}, "tau_h and tau_l"),
    ({"T_sim": math.inf}, "must be finite"),
    ({"D_h": math.nan}, "must be finite"),
    ({"z_sea": math.nan}, "must be finite"),
    ({"max_steps": -1}, "negative"),
    ({"cols_per_lane": 3}, "cols_per_lane"),
    ({"seg_rows": -8}, "seg_rows"),
    ({"inflow_cell": 5, "inflow_peak": math.nan}, "inflow"),
]


@pytest.mark.parametrize("fields,msg", BAD, ids=[",".join(f) + f"-{i}" for i, (f, _) in enumerate(BAD)])
def test_create_rejects_bad_config(fields, msg):
    L = lib.core()
    s = C.c_void_p(123)
    c = _cfg(**fields)
    assert L.fcab_sim_create(C.byref(s), C.byref(c), None) == -1
    assert not s.value                     # no session handed out
    assert msg in L.fcab_last_error().decode()


@pytest.mark.parametrize("double", [False, True])
def test_dropin_run_rejects_bad_run_config(double):
    d, p, _, _ = load_case(GOLDEN / "tiny_3x3.npz")
    for field, value, want in (("U", 0, -2), ("K", 5, -2), ("dt_max", 0.0, -2),
                               ("dx", math.nan, -2)):
        g = DropinGrid(d, p, double=double)
        setattr(g.cfg.phys, field, value)
        assert g.run() == want, field
    g = DropinGrid(d, p, double=double)
    g.cfg.block_x, g.cfg.block_y = 7, 3
    assert g.run() == -1
    g = DropinGrid(d, p, double=double)
    g.g.nrows = 0
    assert g.run() == -2
