"""Host side of the row-split runs (floodca_b200.slabs), on the CPU: the slab
ranges and slab rasters, and the per-rank driver (max-reduction of the
velocity maximum, halo exchange with both neighbours, the step loop) on
gloo ranks. The slabs here are stand-ins with the same interface as the
device slabs: a stencil that reads three rows each way and a step size set
by the global maximum, so a wrong halo row, a missing exchange or a local
instead of a global maximum changes the result."""
import multiprocessing as mp
import socket
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from floodca_b200 import synth
from floodca_b200.slabs import HALO, RankSlab, SlabSpec, run_slabs, slab_domain, slab_specs


def test_slab_specs_cover_rows():
    for nr, parts in [(10, 3), (4096, 4), (97, 8), (3, 1), (6, 2)]:
        sp = slab_specs(nr, parts)
        assert sp[0].r0 == 0 and sp[-1].r1 == nr
        assert all(a.r1 == b.r0 for a, b in zip(sp, sp[1:]))
        assert all(s.rows >= HALO for s in sp) or parts == 1
        assert sp[0].hn == 0 and sp[-1].hs == 0
        assert all(s.hn == HALO for s in sp[1:]) and all(s.hs == HALO for s in sp[:-1])
    with pytest.raises(ValueError):
        slab_specs(5, 2)


def test_slab_domain_rows_edges_inflow():
    d, p = synth.config1(n=64)
    nc = d.shape[1]
    p = p.with_(edges=(1, 1, 1, 0), inflow_cell=20 * nc + 7)
    sp = slab_specs(64, 3)                       # rows [0,21) [21,42) [42,64)
    d0, p0 = slab_domain(d, p, sp[0])
    assert d0.shape == (21 + HALO, nc) and np.array_equal(d0.z, d.z[:24])
    assert p0.edges == (1, 0, 1, 0) and p0.inflow_cell == 20 * nc + 7
    d1, p1 = slab_domain(d, p, sp[1])
    assert d1.shape == (21 + 2 * HALO, nc) and np.array_equal(d1.h, d.h[18:45])
    assert p1.edges == (0, 0, 1, 0)
    assert p1.inflow_cell == (20 - 18) * nc + 7   # in the north halo
    d2, p2 = slab_domain(d, p, sp[2])
    assert p2.edges == (0, 1, 1, 0) and p2.inflow_cell == -1
    assert np.array_equal(d2.mask, d.mask[39:])


# ---------------------------------------------------------------------------
# Stand-in slabs for the gloo driver test.

class ToySlab:
    """rows x nc float64 field plus halo rows; step: x += dt * (x[i-3] +
    x[i+3] + x[i-1] + x[i+1] - 4 x[i]) * w(i), dt = 0.05 / (1 + max |x|)
    over the whole domain."""

    def __init__(self, full: np.ndarray, spec: SlabSpec, steps: int):
        self.spec = spec
        self.nc = full.shape[1]
        a, b = spec.r0 - spec.hn, spec.r1 + spec.hs
        self.x = full[a:b].copy()
        self.vmax = torch.zeros(1, dtype=torch.int64)
        self.dt = 0.0
        self.n = 0
        self.steps = steps
        self.pending = True
        self._publish()

    def _own(self):
        return self.x[self.spec.hn:self.spec.hn + self.spec.rows]

    def _publish(self):
        m = float(np.abs(self._own()).max())
        self.vmax[0] = int(np.array(m, np.float64).view(np.int64))

    def stream(self):
        return None

    def finalize(self):
        if self.pending and self.n < self.steps:
            m = float(np.array(int(self.vmax[0]), np.int64).view(np.float64))
            self.dt = 0.05 / (1.0 + m)
        self.pending = False

    def step(self):
        if self.n >= self.steps:
            return
        x = np.pad(self.x, ((3, 3), (0, 0)))
        hn, r = self.spec.hn, self.spec.rows
        i = np.arange(hn, hn + r) + 3
        w = 1.0 + 0.1 * np.arange(self.nc)[None, :] / self.nc
        lap = x[i - 3] + x[i + 3] + x[i - 1] + x[i + 1] - 4 * x[i]
        self.x[hn:hn + r] = x[i] + self.dt * lap * w
        self.n += 1
        self.pending = True
        self._publish()

    def poll(self):
        return SimpleNamespace(done=self.n >= self.steps and not self.pending)

    def rows_buffer(self, n):
        return torch.empty((n, self.nc), dtype=torch.float64)

    def rows_get(self, row0, buf):
        a = self.spec.hn + row0
        buf.copy_(torch.from_numpy(self.x[a:a + buf.shape[0]]))

    def rows_put(self, row0, buf):
        a = self.spec.hn + row0
        self.x[a:a + buf.shape[0]] = buf.numpy()


def _toy_field(nr, nc):
    rng = np.random.default_rng(5)
    return rng.uniform(0, 1, (nr, nc))


def _toy_single(nr, nc, steps):
    s = ToySlab(_toy_field(nr, nc), SlabSpec(0, nr, 0, 0), steps)
    for _ in range(steps + 1):
        s.finalize()
        s.step()
    return s.x


def _gloo_rank(rank, world, port, nr, nc, steps, q):
    import os
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    spec = slab_specs(nr, world)[rank]
    comm = RankSlab(ToySlab(_toy_field(nr, nc), spec, steps), rank, world, staged=True)
    it = run_slabs(comm, check_every=7)
    s = comm.slabs[0]
    q.put((rank, spec.r0, s._own().copy(), it))
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_rank_slabs_gloo_equal_single_domain(world):
    nr, nc, steps = 23, 9, 40
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_gloo_rank, args=(r, world, port, nr, nc, steps, q))
          for r in range(world)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    got = np.concatenate([r[2] for r in res])
    ref = _toy_single(nr, nc, steps)
    assert np.array_equal(got, ref)
    assert len({r[3] for r in res}) == 1          # every rank stopped at the same iteration


def test_toy_detects_a_missing_exchange():
    """The stand-in is sensitive to the halo: slabs that never exchange
    differ from the single domain."""
    nr, nc, steps = 23, 9, 10
    sp = slab_specs(nr, 2)
    slabs = [ToySlab(_toy_field(nr, nc), s, steps) for s in sp]
    for _ in range(steps + 1):
        for s in slabs:
            s.finalize()
            s.step()
    got = np.concatenate([s._own() for s in slabs])
    assert not np.array_equal(got, _toy_single(nr, nc, steps))


def test_merge_stats_counts_inflow_once():
    a = dict(t=10.0, dt_base=1.0, step=5, done=1, V=3.0, V0=1.0, V_rain=1.5, clamp_err=0.0,
             V_sea=0.25, V_bnd=0.25, V_in=2.0, cap_active=3, cap_total=10, dt_min_hits=1,
             E_mass=0.0, dt_full_passes=2)
    b = dict(a, V=2.0, V0=0.5, V_rain=0.5, V_sea=0.0, V_bnd=0.0, cap_active=1, cap_total=6)
    from floodca_b200.slabs import merge_stats
    m = merge_stats([a, b], [False, True])          # b owns the inflow cell
    assert (m["V"], m["V0"], m["V_rain"], m["cap_active"], m["cap_total"]) == (5.0, 1.5, 2.0, 4, 16)
    assert m["V_in"] == 2.0 and (m["step"], m["t"], m["dt_min_hits"]) == (5, 10.0, 1)
    # V + V_sea + V_bnd - V_rain - V_in - V0 = 5 + 0.5 - 2 - 2 - 1.5 = 0
    assert m["E_mass"] == 0.0
