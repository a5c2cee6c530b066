"""Host <-> device copies of the sessions (pinned staging, several host
threads): what is uploaded comes back unchanged, for grids of one chunk,
many uneven chunks spread over the workers, and rows wider than a staging
slot."""
import numpy as np
import pytest

from floodca_b200 import abi
from floodca_b200.sim import Domain, RunParams, Session

pytestmark = pytest.mark.gpu


def _random_domain(nr, nc, dtype, seed):
    rng = np.random.default_rng(seed)
    f = lambda lo, hi: rng.uniform(lo, hi, (nr, nc)).astype(dtype)
    mask = np.full((nr, nc), abi.FCA_LAND, np.uint8)
    mask[rng.uniform(size=(nr, nc)) < 0.05] = abi.FCA_WALL
    return Domain(z=f(0, 50), mask=mask, n=f(0.02, 0.1), C=f(0, 1), Rday=f(0, 0.1),
                  h=f(0, 2), dx=30.0, hmax=f(2, 3), tmax=f(0, 100))


@pytest.mark.parametrize("nr,nc,prec", [
    (5, 7, "f32"), (3000, 1531, "f32"), (3000, 1531, "f64"), (1, 1_200_000, "f32"),
    (700_001, 3, "f32"), (1023, 4097, "f64")])
def test_upload_download_round_trip(nr, nc, prec):
    dt = np.float64 if prec == "f64" else np.float32
    d = _random_domain(nr, nc, dt, nr + nc)
    with Session(d, RunParams(steps=1), precision=prec) as s:
        h, hmax, tmax = s.download()
        assert np.array_equal(h, d.h) and np.array_equal(hmax, d.hmax)
        assert np.array_equal(tmax, d.tmax)
        # a second upload of new state through the same staging buffers
        h2 = (d.h * 0.5).astype(dt)
        s.L.fcab_sim_upload_state(s.h, h2.ctypes.data, None, None)
        s.L.fcab_sim_reset_time(s.h, 0.0, 0, 0.0, -1)
        h, hmax, tmax = s.download()
        assert np.array_equal(h, h2) and np.array_equal(hmax, h2)
        assert not tmax.any()


def test_session_buffers_are_reused_and_released():
    """A destroyed session's buffers serve the next session of the same
    size (no new device memory), hold no stale state, and
    fcab_release_cached_memory frees them."""
    import torch

    from floodca_b200.lib import core
    d = _random_domain(2000, 2000, np.float32, 1)
    p = RunParams(steps=10)
    with Session(d, p) as s:
        s.run()
        h_ref = s.download()[0]
    free_cached = torch.cuda.mem_get_info()[0]
    with Session(d, p) as s:
        free_during = torch.cuda.mem_get_info()[0]
        s.run()
        assert np.array_equal(s.download()[0], h_ref)
    assert abs(free_during - free_cached) < (8 << 20)      # the cached blocks, reused
    core().fcab_release_cached_memory()
    assert torch.cuda.mem_get_info()[0] - free_cached > (100 << 20)   # ~150 MB freed
