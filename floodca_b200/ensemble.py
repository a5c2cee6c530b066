"""Batched ensembles of WCA runs (config 4: 256 members of side 512-2048) and
their one-at-a-time baseline.

Config 4: members of side drawn uniformly from 512..2048 (multiples of 64),
each with its own seeded terrain (the config-1 generator), Manning n scaled
by lognormal(0, 0.3), uniform rain of 20-150 mm/h for 0.5-4 h, 8 h
simulated, open south edge, 10-minute output windows, independent adaptive
dt per member.

`run_batched` advances every member together (fcab_batch_*: one launch per
ensemble step, CUDA graphs of launches, members either running freely to
their ends or paced by output windows); `run_one_at_a_time` runs the
same members with the same kernel one after another, the way the reference
runs scenarios (src/hybrid/main_ens_mpi_cuda.c:69-120). Both report
members/hour. The tile shape (columns per lane, rows per work unit) comes
from `autotune`, which times short batched runs on a sample of members and
caches the choice in a JSON file.
"""
from __future__ import annotations

import ctypes as C
import json
import time
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import synth
from .abi import FcabBatchInfo
from .lib import check, core
from .sim import Domain, RunParams, Session

TUNING_FILE = Path(__file__).resolve().parent / "tuning.json"


@dataclass
class Member:
    side: int
    seed: int
    n_scale: float
    rain_mm_h: float
    rain_h: float
    T_sim: float = 8 * 3600.0

    def params(self) -> RunParams:
        return synth.south_open().with_(T_sim=self.T_sim, hyeto="uniform",
                                        rain_end=self.rain_h * 3600.0)


def config4_members(n: int = 256, seed: int = 4, sides=(512, 2048), T_sim: float = 8 * 3600.0,
                    rain=(20.0, 150.0), dur=(0.5, 4.0)) -> list[Member]:
    rng = np.random.default_rng(seed)
    choices = np.arange(sides[0], sides[1] + 1, 64)
    return [Member(side=int(rng.choice(choices)), seed=int(seed * 100000 + i),
                   n_scale=float(rng.lognormal(0.0, 0.3)),
                   rain_mm_h=float(rng.uniform(*rain)), rain_h=float(rng.uniform(*dur)),
                   T_sim=T_sim) for i in range(n)]


# ---------------------------------------------------------------------------
# Terrain on the GPU (same recipe as synth.make_terrain: plane sloping south,
# fBm relief spanning [-A, A], a 3-cell channel 2 m deep, six Voronoi
# Manning classes), used to set up large ensembles quickly.

def terrain_torch(side: int, seed: int, amplitude: float = 5.0, dx: float = 90.0,
                  slope: float = 0.005, hurst: float = 0.7, n_scale: float = 1.0,
                  device="cuda"):
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    nr = nc = side
    ky = torch.fft.fftfreq(nr, device=device, dtype=torch.float64)[:, None]
    kx = torch.fft.rfftfreq(nc, device=device, dtype=torch.float64)[None, :]
    k = torch.sqrt(kx * kx + ky * ky)
    k[0, 0] = 1.0
    amp = k ** (-(hurst + 1.0))
    amp[0, 0] = 0.0
    phase = torch.rand(amp.shape, generator=g, device=device, dtype=torch.float64) * (2 * np.pi)
    f = torch.fft.irfft2(amp * torch.exp(1j * phase), s=(nr, nc))
    f = f - f.mean()
    f = f * (amplitude / f.abs().max())
    rows = torch.arange(nr, device=device, dtype=torch.float64)[:, None]
    z = 10.0 + slope * dx * (nr - 1 - rows) + f
    c0 = nc // 2 - 1
    z[:, c0:c0 + 3] -= 2.0
    nseed = max(8, nr * nc // 4096)
    pts = torch.rand((nseed, 2), generator=g, device=device, dtype=torch.float32)
    pts = pts * torch.tensor([nr, nc], device=device, dtype=torch.float32)
    cls = torch.randint(0, len(synth.MANNING_CLASSES), (nseed,), generator=g, device=device)
    yy = torch.arange(nr, device=device, dtype=torch.float32) + 0.5
    xx = torch.arange(nc, device=device, dtype=torch.float32) + 0.5
    best = torch.empty((nr, nc), dtype=torch.long, device=device)
    step = max(1, (1 << 24) // (nc * nseed))
    for r0 in range(0, nr, step):
        r1 = min(nr, r0 + step)
        q = torch.stack(torch.meshgrid(yy[r0:r1], xx, indexing="ij"), -1).reshape(-1, 2)
        best[r0:r1] = torch.cdist(q, pts).argmin(1).reshape(r1 - r0, nc)
    manning = torch.tensor(synth.MANNING_CLASSES, device=device, dtype=torch.float64)
    n = manning[cls[best]] * n_scale
    return z.float().contiguous(), n.float().contiguous()


def member_session(m: Member, math: str = "exact", h_init: float = 0.0,
                   device="cuda") -> Session:
    """A session for one member, uploaded from device tensors (initial depth
    h_init everywhere; 0 for the member as specified)."""
    import torch
    z, n = terrain_torch(m.side, m.seed, n_scale=m.n_scale, device=device)
    shape = (m.side, m.side)
    h = torch.full(shape, h_init, device=device, dtype=torch.float32)
    rday = torch.full(shape, m.rain_mm_h * 24.0 / 1000.0, device=device, dtype=torch.float32)
    ones = torch.ones(shape, device=device, dtype=torch.float32)
    mask = torch.zeros(shape, device=device, dtype=torch.uint8)
    torch.cuda.synchronize()
    s = Session.from_device(shape, 90.0, m.params(), z, h, mask, n=n, Cf=ones, Rday=rday,
                            precision="f32", math=math)
    return s


def member_domain(m: Member) -> tuple[Domain, RunParams]:
    """The member as host arrays (for checks against the oracle)."""
    z, n = terrain_torch(m.side, m.seed, n_scale=m.n_scale)
    shape = (m.side, m.side)
    d = Domain(z=z.cpu().numpy(), mask=np.zeros(shape, np.uint8), n=n.cpu().numpy(),
               C=np.ones(shape, np.float32),
               Rday=np.full(shape, m.rain_mm_h * 24.0 / 1000.0, np.float32),
               h=np.zeros(shape, np.float32), dx=90.0)
    return d, m.params()


# ---------------------------------------------------------------------------

class Batch:
    """fcab_batch_* over uploaded FP32 sessions. member_seg: rows per work
    unit for each member (None: seg_rows for all)."""

    def __init__(self, sessions: list[Session], cols_per_lane: int = 0, seg_rows: int = 0,
                 member_seg=None):
        self.L = core()
        self.sessions = sessions
        arr = (C.c_void_p * len(sessions))(*[s.h.value for s in sessions])
        segs = None if member_seg is None else (C.c_int * len(sessions))(*member_seg)
        b = C.c_void_p()
        check(self.L.fcab_batch_create(C.byref(b), arr, len(sessions), cols_per_lane, seg_rows,
                                       segs, None), "fcab_batch_create")
        self.b = b

    def run(self, window: float = 600.0, graph_steps: int = 16, max_windows: int = 0) -> None:
        check(self.L.fcab_batch_run(self.b, window, graph_steps, max_windows), "fcab_batch_run")

    def info(self) -> dict:
        i = FcabBatchInfo()
        check(self.L.fcab_batch_info(self.b, C.byref(i)), "fcab_batch_info")
        return {f[0]: getattr(i, f[0]) for f in i._fields_}

    def close(self):
        if self.b:
            self.L.fcab_batch_destroy(self.b)
            self.b = None


def _sync():
    import torch
    torch.cuda.synchronize()


DEFAULT_TUNING = {"cols_per_lane": 2, "seg_rows_by_class": [[0, 1 << 30, 64]]}


def seg_for(side: int, tuning: dict) -> int:
    for lo, hi, seg in tuning["seg_rows_by_class"]:
        if lo <= side <= hi:
            return int(seg)
    return 64


THRESHOLDS = (0.10, 0.25, 0.50)
ROW_FIELDS = ("member", "side", "seed", "n_scale", "rain_mm_h", "rain_h", "rank", "steps",
              "sim_time_s", "rain_volume_m3", "boundary_volume_m3", "mass_err_rel",
              "flooded_cells_010", "flooded_cells_025", "flooded_cells_050", "max_depth_m")


def member_row(idx: int, m: Member, s: Session, rank: int = 0) -> dict:
    """One member's summary in the layout of the reference ensemble's
    per-scenario CSV (src/hybrid/ens_common.c:223-258): steps, simulated
    time, rain volume, mass-balance error, flooded cells at 0.10 / 0.25 /
    0.50 m and the largest peak depth."""
    st = s.stats()
    fl, mx = s.count_flooded(THRESHOLDS)
    return {"member": idx, "side": m.side, "seed": m.seed, "n_scale": m.n_scale,
            "rain_mm_h": m.rain_mm_h, "rain_h": m.rain_h, "rank": rank, "steps": st["step"],
            "sim_time_s": st["t"], "rain_volume_m3": st["V_rain"],
            "boundary_volume_m3": st["V_bnd"], "mass_err_rel": st["E_mass"],
            "flooded_cells_010": fl[0], "flooded_cells_025": fl[1], "flooded_cells_050": fl[2],
            "max_depth_m": mx}


def write_rows(path, rows: list[dict]) -> None:
    with open(path, "w") as f:
        f.write(",".join(ROW_FIELDS) + "\n")
        for r in sorted(rows, key=lambda r: r["member"]):
            f.write(",".join(str(r[k]) for k in ROW_FIELDS) + "\n")


def gather_rows(rows: list[dict]) -> list[dict]:
    """Every rank's member rows, on every rank (one host gather after the
    run: the only collective of the sharded ensemble)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return list(rows)
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, list(rows))
    return sorted((r for part in out for r in part), key=lambda r: r["member"])


def run_batched(members: list[Member], math="exact", tuning: dict | None = None,
                window=0.0, graph_steps=16, collect=False, ids=None, rank: int = 0) -> dict:
    """All members in one batch; window > 0 paces them by output windows.
    ids: the members' indices in the whole ensemble (for the rows)."""
    tuning = tuning or DEFAULT_TUNING
    t0 = time.perf_counter()
    sessions = [member_session(m, math) for m in members]
    _sync()
    t_setup = time.perf_counter() - t0
    b = Batch(sessions, tuning["cols_per_lane"], 0, [seg_for(m.side, tuning) for m in members])
    _sync()
    t1 = time.perf_counter()
    b.run(window, graph_steps)
    _sync()
    wall = time.perf_counter() - t1
    stats = [s.stats() for s in sessions]
    ids = list(range(len(members))) if ids is None else list(ids)
    out = {"members": len(members), "wall_s": wall, "setup_s": t_setup,
           "members_per_hour": len(members) / wall * 3600.0, "info": b.info(),
           "cell_steps": sum(st["step"] * m.side * m.side for st, m in zip(stats, members)),
           "stats": stats,
           "rows": [member_row(i, m, s, rank) for i, m, s in zip(ids, members, sessions)]}
    if collect:
        out["hmax"] = [s.download()[1] for s in sessions]
    b.close()
    for s in sessions:
        s.close()
    return out


def run_one_at_a_time(members: list[Member], math="exact", collect=False) -> dict:
    """The same kernel, one member after another (each its own session)."""
    stats, hmax, wall, setup = [], [], 0.0, 0.0
    for m in members:
        t0 = time.perf_counter()
        s = member_session(m, math)
        _sync()
        t1 = time.perf_counter()
        s.run()
        _sync()
        wall += time.perf_counter() - t1
        setup += t1 - t0
        stats.append(s.stats())
        if collect:
            hmax.append(s.download()[1])
        s.close()
    out = {"members": len(members), "wall_s": wall, "setup_s": setup,
           "members_per_hour": len(members) / wall * 3600.0, "stats": stats,
           "cell_steps": sum(st["step"] * m.side * m.side for st, m in zip(stats, members))}
    if collect:
        out["hmax"] = hmax
    return out


def shard(members: list[Member], rank: int, world: int) -> list[int]:
    """Indices of the members rank `rank` of `world` runs: longest-first
    greedy assignment by cell count (members are independent, so ranks share
    nothing on the data path)."""
    order = sorted(range(len(members)), key=lambda i: (-members[i].side, i))
    load = [0] * world
    mine = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += members[i].side ** 2
        mine[r].append(i)
    return sorted(mine[rank])


# ---------------------------------------------------------------------------
# Autotuner. Columns per lane (strip width, a template parameter shared by the
# whole batch) and rows per work unit (tile height, chosen per member size
# class) are timed on batches of sample members of each size class, started
# wet (0.05 m everywhere, so every step does the full face work) and run for
# a fixed simulated span. The column width minimising the ensemble's
# estimated time (class cell counts / class throughput) wins; each class then
# takes its fastest tile height at that width. Cached per GPU, math mode and
# size classes.

CPL_CHOICES = (1, 2, 4)
SEG_CHOICES = (32, 64, 128)
SIZE_CLASSES = ((0, 1023), (1024, 1535), (1536, 1 << 30))


def _tuning_key(math: str) -> str:
    import torch
    return f"{torch.cuda.get_device_name()}|{math}|" + ",".join(f"{a}-{b}" for a, b in SIZE_CLASSES)


def choose_tuning(trials: list[dict], work_by_class: dict) -> dict:
    """From trials [{cls, cpl, seg, rate}] (rate in cell-steps/s) and the
    cells of each class, the width with the least estimated time and each
    class's best height at that width."""
    best_t, best = None, None
    for cpl in sorted({t["cpl"] for t in trials}):
        est, segs = 0.0, []
        for ci, (lo, hi) in enumerate(SIZE_CLASSES):
            if work_by_class.get(ci, 0) == 0:
                continue
            cand = [t for t in trials if t["cls"] == ci and t["cpl"] == cpl]
            if not cand:
                est = float("inf")
                break
            top = max(cand, key=lambda t: t["rate"])
            est += work_by_class[ci] / top["rate"]
            segs.append([lo, hi, top["seg"]])
        if best_t is None or est < best_t:
            best_t, best = est, {"cols_per_lane": cpl, "seg_rows_by_class": segs}
    return best


def autotune(members: list[Member], math="exact", per_class: int = 6, windows: int = 2,
             window: float = 600.0, cache: Path | None = TUNING_FILE,
             force: bool = False) -> dict:
    key = _tuning_key(math)
    table = {}
    if cache and cache.exists():
        table = json.loads(cache.read_text())
        if key in table and not force:
            return table[key]
    rng = np.random.default_rng(0)
    trials, work = [], {}
    for ci, (lo, hi) in enumerate(SIZE_CLASSES):
        idx = [i for i, m in enumerate(members) if lo <= m.side <= hi]
        if not idx:
            continue
        work[ci] = sum(members[i].side ** 2 for i in idx)
        pick = [members[i] for i in sorted(rng.choice(idx, min(per_class, len(idx)),
                                                      replace=False))]
        for cpl in CPL_CHOICES:
            for seg in SEG_CHOICES:
                sessions = [member_session(m, math, h_init=0.05) for m in pick]
                b = Batch(sessions, cpl, seg)
                _sync()
                t0 = time.perf_counter()
                b.run(window=window, graph_steps=16, max_windows=windows)
                _sync()
                dt = time.perf_counter() - t0
                cells = sum(s.stats()["step"] * m.side * m.side for s, m in zip(sessions, pick))
                trials.append({"cls": ci, "cpl": b.info()["cols_per_lane"], "seg": seg,
                               "rate": cells / dt})
                b.close()
                for s in sessions:
                    s.close()
    res = choose_tuning(trials, work)
    res["trials"] = trials
    if cache:
        table[key] = res
        cache.write_text(json.dumps(table, indent=1) + "\n")
    return res


# ---------------------------------------------------------------------------

def main(argv=None) -> int:
    """Config-4 ensemble: batched vs one-at-a-time members/hour.

    python -m floodca_b200.ensemble [--members 256] [--baseline-members 16]
    Under torchrun each rank runs its shard of the members (no collective on
    the data path); the wall time is the max over ranks.
    """
    import argparse
    import os
    ap = argparse.ArgumentParser()
    ap.add_argument("--members", type=int, default=256)
    ap.add_argument("--baseline-members", type=int, default=16,
                    help="members timed one at a time (a seeded subsample)")
    ap.add_argument("--math", default="exact")
    ap.add_argument("--hours", type=float, default=8.0)
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--tuning-cache", default=str(TUNING_FILE))
    ap.add_argument("--retune", action="store_true")
    ap.add_argument("--paced", action="store_true", help="also time the 10-minute paced run")
    ap.add_argument("--out", default="")
    ap.add_argument("--csv", default="", help="per-member rows (rank 0 writes all ranks')")
    a = ap.parse_args(argv)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    members = config4_members(a.members, T_sim=a.hours * 3600.0)
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl")
    mine = shard(members, rank, world)
    local = [members[i] for i in mine]
    tune = DEFAULT_TUNING if a.no_tune else autotune(members, a.math,
                                                     cache=Path(a.tuning_cache),
                                                     force=a.retune)
    bat = run_batched(local, a.math, tune, window=0.0, ids=mine, rank=rank)
    wall = bat["wall_s"]
    rows = gather_rows(bat["rows"])
    if world > 1:
        import torch
        import torch.distributed as dist
        w = torch.tensor([wall, float(bat["cell_steps"])], device="cuda", dtype=torch.float64)
        mx = w.clone()
        dist.all_reduce(mx[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(w[1:], op=dist.ReduceOp.SUM)
        wall, total_cells = float(mx[0]), float(w[1])
    else:
        total_cells = float(bat["cell_steps"])
    res = {"workload": f"config 4: {a.members} members, side 512..2048 step 64, "
                       f"{a.hours:g} h simulated, out_every 600 s",
           "n_gpus": world,
           "tuning": {k: tune[k] for k in ("cols_per_lane", "seg_rows_by_class")},
           "batched": {"members": a.members, "wall_s": wall,
                       "members_per_hour": a.members / wall * 3600.0,
                       "gcell_steps_per_s": total_cells / wall / 1e9,
                       "setup_s_rank0": bat["setup_s"], "info_rank0": bat["info"]}}
    if rank == 0:
        res["members_rows"] = len(rows)
        if a.csv:
            write_rows(a.csv, rows)
        if a.paced:
            paced = run_batched(local, a.math, tune, window=600.0)
            res["batched_paced_600s_rank0"] = {
                "wall_s": paced["wall_s"], "info": paced["info"],
                "steps_and_time_equal": all(x["step"] == y["step"] and x["t"] == y["t"]
                                            for x, y in zip(bat["stats"], paced["stats"]))}
        # one at a time on a seeded uniform subsample of this rank's members:
        # its mean wall time per member estimates the ensemble's
        rng = np.random.default_rng(1)
        idx = sorted(rng.choice(len(local), min(a.baseline_members, len(local)), replace=False))
        one = run_one_at_a_time([local[i] for i in idx], a.math)
        res["one_at_a_time_1gpu"] = {
            "members": len(idx), "wall_s": one["wall_s"],
            "members_per_hour": one["members_per_hour"],
            "gcell_steps_per_s": one["cell_steps"] / one["wall_s"] / 1e9,
            "steps_and_time_equal_batched": all(
                one["stats"][j]["step"] == bat["stats"][i]["step"] and
                one["stats"][j]["t"] == bat["stats"][i]["t"] for j, i in enumerate(idx))}
        res["speedup_members_per_hour"] = (res["batched"]["members_per_hour"] /
                                           one["members_per_hour"])
        txt = json.dumps(res, indent=1)
        if a.out:
            Path(a.out).write_text(txt + "\n")
        print(txt)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    import sys
    sys.exit(main())
