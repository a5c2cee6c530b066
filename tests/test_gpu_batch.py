"""Batched ensembles (fcab_batch_*): every member of a batch ends with the
same depth, max depth, time of max depth, step count and simulated time as
the same member run alone in its own session, bit for bit, whatever the mix
of member sizes, parameters and rain; output windows only pace the members.
Each member of the mixed batches is also compared with the compiled
reference core run on its own (FP32 bit for bit), the semantics the batch
replaces being one fca_cuda_ens_run per member (src/cuda/kernels.cu:836-997)."""
import ctypes as C

import numpy as np
import pytest

from floodca_b200 import abi, synth
from floodca_b200.ensemble import Batch, Member, member_session
from floodca_b200.lib import FcabError
from floodca_b200.sim import Session, run_session
from tests import refpin

pytestmark = pytest.mark.gpu


def _members(K=4, rain_field=False, sea=False, seed=11):
    rng = np.random.default_rng(seed)
    out = []
    for i, (nr, nc) in enumerate([(64, 64), (96, 160), (200, 72), (3, 3), (1, 40), (130, 257)]):
        d = synth.make_terrain(synth.TerrainSpec(nr, nc, seed=seed * 10 + i,
                                                 n_scale=float(rng.lognormal(0, 0.3))))
        d, p = synth.box_rain(d, synth.south_open().with_(K=K, T_sim=float(rng.uniform(3600, 7200))),
                              float(rng.uniform(20, 150)), float(rng.choice([0.5, 1.0])))
        d.h = np.full(d.shape, float(rng.uniform(0, 0.05)), np.float32)
        if rain_field:
            d.C = rng.uniform(0.3, 1.0, d.shape).astype(np.float32)
        if sea:                     # every member keeps LAND cells (and its rain field)
            if nr >= 3:
                d.mask[-1:, :] = abi.FCA_SEA
                d.z[-1:, :] = -1.0
            d.mask[:, :1] = abi.FCA_WALL
        out.append((d, p))
    return out


def _result(s):
    h, hmax, tmax = s.download()
    return {**s.stats(), "h": h, "hmax": hmax, "tmax": tmax}


def _check_equal(single, s):
    st = s.stats()
    h, hmax, tmax = s.download()
    assert st["step"] == single["step"] and st["t"] == single["t"], (st, single["step"])
    assert np.array_equal(h, single["h"])
    assert np.array_equal(hmax, single["hmax"])
    assert np.array_equal(tmax, single["tmax"])
    assert st["V"] == pytest.approx(single["V"], rel=1e-12, abs=1e-9)


@pytest.mark.parametrize("K,rain_field,sea,cpl,seg", [
    (4, False, False, 2, 64), (4, False, False, 1, 32), (4, False, False, 4, 128),
    (8, False, False, 2, 64), (8, True, False, 1, 48), (4, True, True, 2, 16),
    (8, False, True, 2, 64)])
def test_batch_equals_single_sessions(K, rain_field, sea, cpl, seg):
    mem = _members(K, rain_field, sea)
    singles = [run_session(d, p) for d, p in mem]
    sessions = [Session(d, p) for d, p in mem]
    b = Batch(sessions, cpl, seg)
    try:
        b.run(window=600.0, graph_steps=8)
        info = b.info()
        assert info["members"] == len(mem) and info["windows"] >= 2
        for single, s, (d, p) in zip(singles, sessions, mem):
            _check_equal(single, s)
            refpin.check_reference(_result(s), d, p)
    finally:
        b.close()
        for s in sessions:
            s.close()


def test_batch_windows_resume():
    """Two windows, then the rest: the same results as one call."""
    mem = _members(4)
    singles = [run_session(d, p) for d, p in mem]
    sessions = [Session(d, p) for d, p in mem]
    b = Batch(sessions)
    try:
        b.run(window=600.0, graph_steps=16, max_windows=2)
        assert b.info()["windows"] == 2
        for s in sessions:
            st = s.stats()
            assert st["t"] <= 1200.0 + 1e-6 and not st["done"]
        b.run(window=600.0, graph_steps=16)
        for single, s in zip(singles, sessions):
            _check_equal(single, s)
    finally:
        b.close()
        for s in sessions:
            s.close()


def test_batch_free_running():
    """No pacing (window <= 0) and a tile height per member: the same results."""
    mem = _members(8, rain_field=True)
    singles = [run_session(d, p) for d, p in mem]
    sessions = [Session(d, p) for d, p in mem]
    b = Batch(sessions, 2, 64, member_seg=[16, 32, 48, 64, 8, 128])
    try:
        b.run(window=0.0, graph_steps=32)
        assert b.info()["windows"] == 0
        for single, s, (d, p) in zip(singles, sessions, mem):
            _check_equal(single, s)
            refpin.check_reference(_result(s), d, p)
    finally:
        b.close()
        for s in sessions:
            s.close()


def test_batch_rejects_mixed_members():
    mem = _members(4)[:2]
    a = Session(*mem[0])
    d, p = mem[1]
    c = Session(d, p.with_(K=8))
    f = Session(d, p, precision="f64")
    try:
        for pair in ([a, c], [a, f]):
            with pytest.raises(FcabError):
                Batch(pair)
    finally:
        for s in (a, c, f):
            s.close()


def test_device_members_equal_host_members():
    """A config-4 member set up from device tensors runs like the same
    terrain uploaded from the host."""
    from floodca_b200.ensemble import member_domain
    m = Member(side=128, seed=7, n_scale=1.2, rain_mm_h=80.0, rain_h=0.5, T_sim=3600.0)
    d, p = member_domain(m)
    single = run_session(d, p)
    s = member_session(m)
    try:
        s.run()
        _check_equal(single, s)
        refpin.check_reference(_result(s), d, p)
    finally:
        s.close()


def test_member_rows_match_downloaded_depths():
    """The per-member rows (reference ensemble CSV layout) agree with each
    member's downloaded peak depth."""
    from floodca_b200.ensemble import THRESHOLDS, run_batched
    ms = [Member(side=128, seed=31 + i, n_scale=1.0, rain_mm_h=60.0 + 40 * i, rain_h=1.0,
                 T_sim=3600.0) for i in range(3)]
    out = run_batched(ms, collect=True, ids=[7, 8, 9])
    for row, hm, st in zip(out["rows"], out["hmax"], out["stats"]):
        assert row["steps"] == st["step"] and row["sim_time_s"] == st["t"]
        for t, key in zip(THRESHOLDS, ("flooded_cells_010", "flooded_cells_025",
                                       "flooded_cells_050")):
            assert row[key] == int((hm.astype(np.float64) >= t).sum())
        assert row["max_depth_m"] == pytest.approx(float(hm.max()), rel=1e-7)
    assert [r["member"] for r in out["rows"]] == [7, 8, 9]
