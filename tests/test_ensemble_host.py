"""Host side of the batched ensemble: the config-4 member generator and the
terrain recipe used to set members up on the device (run here on the CPU)."""
import numpy as np
import pytest
import torch

from floodca_b200 import abi, synth
from floodca_b200.ensemble import config4_members, terrain_torch


def test_config4_members():
    ms = config4_members(256)
    assert len(ms) == 256
    sides = np.array([m.side for m in ms])
    assert sides.min() >= 512 and sides.max() <= 2048 and np.all(sides % 64 == 0)
    assert len(set(sides.tolist())) > 15
    assert len({m.seed for m in ms}) == 256
    ns = np.log([m.n_scale for m in ms])
    assert abs(ns.mean()) < 0.06 and abs(ns.std() - 0.3) < 0.05
    assert all(20 <= m.rain_mm_h <= 150 and 0.5 <= m.rain_h <= 4.0 for m in ms)
    assert config4_members(256) == ms
    p = ms[0].params()
    assert p.edges == (0, 1, 0, 0) and p.boundary == "open" and p.hyeto == "uniform"
    assert p.T_sim == 8 * 3600.0 and p.out_every == 600.0
    assert p.rain_end == pytest.approx(ms[0].rain_h * 3600.0)


def test_terrain_recipe():
    z, n = terrain_torch(64, 5, n_scale=1.5, device="cpu")
    assert z.shape == (64, 64) and z.dtype == torch.float32 and n.dtype == torch.float32
    zz = z.double().numpy()
    # plane falling 0.005 * 90 m per row toward the south, relief within +-5 m
    plane = 10.0 + 0.45 * (63 - np.arange(64))[:, None]
    rel = zz - plane
    rel[:, 31:34] += 2.0
    assert np.abs(rel).max() <= 5.0 + 1e-4 and np.abs(rel).max() > 4.9
    classes = {round(c * 1.5, 6) for c in synth.MANNING_CLASSES}
    assert {round(float(v), 6) for v in np.unique(n.numpy())} <= classes
    z2, n2 = terrain_torch(64, 5, n_scale=1.5, device="cpu")
    assert torch.equal(z, z2) and torch.equal(n, n2)
    assert not torch.equal(z, terrain_torch(64, 6, device="cpu")[0])


def test_batch_info_layout():
    assert abi.FcabBatchInfo.__name__ == "FcabBatchInfo"
    names = [f[0] for f in abi.FcabBatchInfo._fields_]
    assert names == ["members", "cols_per_lane", "seg_rows", "grid", "total_units",
                     "launches", "windows", "graph_replays"]


def test_shard_partitions_members():
    from floodca_b200.ensemble import shard
    ms = config4_members(256)
    for world in (1, 2, 3, 8):
        parts = [shard(ms, r, world) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(256))
        loads = [sum(ms[i].side ** 2 for i in p) for p in parts]
        assert max(loads) - min(loads) <= 2048 ** 2


def _gloo_rank(rank, world, port, q):
    import os
    import torch.distributed as dist
    from floodca_b200.ensemble import config4_members as mk, shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from floodca_b200.ensemble import gather_rows
    mine = shard(mk(64), rank, world)
    got = [None] * world
    dist.all_gather_object(got, mine)
    t = torch.tensor([float(len(mine))])
    dist.all_reduce(t)
    rows = gather_rows([{"member": i, "rank": rank, "steps": 10 + i} for i in mine])
    q.put((rank, got, float(t), rows))
    dist.destroy_process_group()


def test_shard_gloo_two_ranks():
    """Two ranks compute their shards independently; together they cover
    every member once, and the one host gather after the run gives every
    rank all member rows (what the torchrun ensemble relies on)."""
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_gloo_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, total, rows in res:
        assert sorted(got[0] + got[1]) == list(range(64)) and not set(got[0]) & set(got[1])
        assert total == 64.0
        # every rank holds every member's row once, from the rank that ran it
        assert [r["member"] for r in rows] == list(range(64))
        owner = {i: k for k in range(2) for i in got[k]}
        assert all(r["rank"] == owner[r["member"]] and r["steps"] == 10 + r["member"] for r in rows)


def test_choose_tuning():
    from floodca_b200.ensemble import choose_tuning
    trials = []
    rates = {  # (cls, cpl, seg) -> rate
        (0, 1, 32): 10, (0, 1, 64): 12, (0, 2, 32): 14, (0, 2, 64): 13,
        (2, 1, 32): 20, (2, 1, 64): 22, (2, 2, 32): 25, (2, 2, 64): 30,
    }
    for (c, cpl, seg), r in rates.items():
        trials.append({"cls": c, "cpl": cpl, "seg": seg, "rate": r})
    t = choose_tuning(trials, {0: 100, 2: 1000})
    assert t["cols_per_lane"] == 2
    assert t["seg_rows_by_class"] == [[0, 1023, 32], [1536, 1 << 30, 64]]
    from floodca_b200.ensemble import seg_for
    assert seg_for(512, t) == 32 and seg_for(2048, t) == 64 and seg_for(1100, t) == 64


def test_write_rows(tmp_path):
    from floodca_b200.ensemble import ROW_FIELDS, write_rows
    rows = [{k: (i if k == "member" else 0.5) for k in ROW_FIELDS} for i in (2, 0, 1)]
    p = tmp_path / "m.csv"
    write_rows(p, rows)
    lines = p.read_text().splitlines()
    assert lines[0].split(",") == list(ROW_FIELDS)
    assert [ln.split(",")[0] for ln in lines[1:]] == ["0", "1", "2"]
