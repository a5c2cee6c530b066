"""Row-split runs (fcab_sim_set_slab / fcab_sim_slab_* / fcab_sim_rows_*):
a domain run as 2-4 slabs ends with the same depth, max depth, time of max
depth, step count and time as the same domain run whole, bit for bit, with
the volumes summed over slabs within rounding. The slabs run on one GPU,
in one process (device max and device copies between slabs) or in two
processes that exchange through gloo on the host; no kernel waits on
another. The split runs are also compared with the compiled reference core
run on the whole domain (FP32 bit for bit, FP64 within 1e-12 m)."""
import multiprocessing as mp
import socket

import numpy as np
import pytest

from floodca_b200 import abi, synth
from floodca_b200.lib import FcabError
from floodca_b200.sim import run_session
from floodca_b200.slabs import HALO, Slab, run_split_local, slab_specs
from tests import refpin

pytestmark = pytest.mark.gpu


def _domain(nr, nc, K=4, seed=3, rain_field=False, sea=False, U=1, inflow_row=None):
    d = synth.make_terrain(synth.TerrainSpec(nr, nc, seed=seed))
    d, p = synth.box_rain(d, synth.south_open().with_(K=K, U=U, T_sim=5400.0), 60.0, 1.0)
    d.h = np.full(d.shape, 0.01, np.float32)
    if rain_field:
        rng = np.random.default_rng(seed)
        d.C = rng.uniform(0.3, 1.0, d.shape).astype(np.float32)
    if sea:
        d.mask[-2:, :] = abi.FCA_SEA
        d.z[-2:, :] = -1.0
        d.mask[:, :1] = abi.FCA_WALL
        d.mask[nr // 2, nc // 3:nc // 2] = abi.FCA_WALL
    if inflow_row is not None:
        p = p.with_(inflow_cell=inflow_row * nc + nc // 2, inflow_peak=40.0,
                    inflow_t_peak=1800.0, inflow_t_end=3600.0)
    return d, p


def _check_equal(single, split, rel=1e-11):
    assert split["step"] == single["step"] and split["t"] == single["t"]
    assert split["dt_base"] == single["dt_base"]
    assert np.array_equal(split["h"], single["h"])
    assert np.array_equal(split["hmax"], single["hmax"])
    assert np.array_equal(split["tmax"], single["tmax"])
    for k in ("V", "V0", "V_rain", "V_in", "V_sea", "V_bnd", "clamp_err"):
        assert split[k] == pytest.approx(single[k], rel=rel, abs=1e-6), k
    assert split["cap_active"] == single["cap_active"]
    assert split["cap_total"] == single["cap_total"]
    assert split["dt_min_hits"] == single["dt_min_hits"]
    # the seeded dt pruning deferred the same steps to the full pass
    assert split["dt_full_passes"] == single["dt_full_passes"]
    assert split["E_mass"] < 1e-6


@pytest.mark.parametrize("parts,kw", [
    (2, dict(K=4)),
    (2, dict(K=4, inflow_row=None)),
    (3, dict(K=8, rain_field=True, sea=True)),
    (4, dict(K=4, U=2, sea=True)),
])
def test_split_equals_whole_domain(parts, kw):
    nr, nc = 150, 130
    if "inflow_row" in kw:
        kw = dict(kw, inflow_row=slab_specs(nr, parts)[1].r0 - 1)   # in the next slab's halo
    d, p = _domain(nr, nc, **kw)
    single = run_session(d, p)
    split = run_split_local(d, p, parts)
    _check_equal(single, split)
    refpin.check_reference(split, d, p)


@pytest.mark.parametrize("K", [4, 8])
def test_split_deferred_dt(K):
    """Dry terrain with a few one-cell water columns, one at a slab edge:
    each column empties in about one step, so the velocity maximum falls
    far below the seed and the seeded pruning defers dt to the full pass,
    on every slab alike."""
    nr, nc = 90, 64
    d, p = _domain(nr, nc, K=K)
    d.h = np.zeros(d.shape, np.float32)
    for r, c, depth in ((10, 10, 3.0), (29, 40, 2.0), (30, 20, 1.2), (60, 50, 0.7)):
        d.h[r, c] = depth
    d.Rday = np.zeros_like(d.h)
    p = p.with_(T_sim=900.0)
    single = run_session(d, p)
    assert single["dt_full_passes"] > 0
    split = run_split_local(d, p, 3)                    # slab edges at rows 30 and 60
    _check_equal(single, split)
    refpin.check_reference(split, d, p)


@pytest.mark.parametrize("precision", ["f64", "f32all"])
def test_split_precisions(precision):
    d, p = _domain(96, 70, K=8, inflow_row=47)
    single = run_session(d, p, precision=precision)
    split = run_split_local(d, p, 2, precision=precision)
    # f32all accumulates the volumes in float
    _check_equal(single, split, rel=1e-5 if precision == "f32all" else 1e-11)
    if precision == "f64":
        refpin.check_reference(split, d, p, kind="f64")


def test_split_cols_per_lane_and_segments():
    """Other launch shapes of the slabs (1- and 4-column lanes, short
    segments) give the same results."""
    d, p = _domain(200, 300, K=4, inflow_row=99)
    single = run_session(d, p)
    ref = refpin.reference(d, p)
    for cpl, seg in ((1, 8), (4, 64)):
        split = run_split_local(d, p, 2, cols_per_lane=cpl, seg_rows=seg)
        _check_equal(single, split)
        refpin.check(split, ref)


def test_rows_round_trip_and_bounds():
    import torch
    d, p = _domain(40, 50)
    spec = slab_specs(40, 2)[1]
    s = Slab(d, p, spec)
    try:
        buf = s.rows_buffer(HALO)
        s.rows_get(-HALO, buf)                        # the north halo as uploaded
        a = spec.r0 - HALO
        assert np.array_equal(buf.cpu().numpy(), d.h[a:a + HALO].astype(np.float32))
        pat = torch.arange(HALO * 50, dtype=torch.float32, device="cuda").reshape(HALO, 50)
        s.rows_put(-HALO, pat)
        out = s.rows_buffer(HALO)
        s.rows_get(-HALO, out)
        torch.cuda.synchronize()
        assert torch.equal(out, pat)
        for row0, n in ((-HALO - 1, 1), (spec.rows, 1)):    # beyond the halo rows
            with pytest.raises(FcabError):
                s.rows_get(row0, s.rows_buffer(n))
        with pytest.raises(FcabError):
            s.advance(1)                              # slabs step through slab_step only
        assert s.vmax.data_ptr() != 0 and s.vmax.dtype == torch.int64
        assert s.info()["land_only"] == 1     # all LAND with its halo: the mask-free kernel
    finally:
        s.close()


def _gloo_rank(rank, world, port, q):
    import os

    import torch
    import torch.distributed as dist

    from floodca_b200.slabs import RankSlab, merge_stats, run_slabs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    torch.cuda.set_device(0)
    d, p = _domain(120, 90, K=8, inflow_row=59)
    spec = slab_specs(120, world)[rank]
    s = Slab(d, p, spec)
    run_slabs(RankSlab(s, rank, world, staged=True), check_every=16)
    h, hmax, tmax = s.download()
    st = s.stats()
    got = [None] * world
    dist.all_gather_object(got, (rank, h, hmax, tmax, st, s.owns_inflow))
    s.close()
    dist.destroy_process_group()
    if rank == 0:
        got.sort(key=lambda g: g[0])
        out = {k: np.concatenate([g[i] for g in got]) for i, k in ((1, "h"), (2, "hmax"), (3, "tmax"))}
        out.update(merge_stats([g[4] for g in got], [g[5] for g in got]))
        q.put(out)


def test_rank_slabs_two_processes_gloo():
    """Two processes, one slab each, halo rows and the velocity maximum
    exchanged through gloo on the host (the NCCL path's driver with host
    staging): the same results as the whole domain."""
    d, p = _domain(120, 90, K=8, inflow_row=59)
    single = run_session(d, p)
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_gloo_rank, args=(r, 2, port, q)) for r in range(2)]
    for pr in ps:
        pr.start()
    out = q.get(timeout=300)
    for pr in ps:
        pr.join(timeout=120)
        assert pr.exitcode == 0
    _check_equal(single, out)
    refpin.check_reference(out, d, p)
