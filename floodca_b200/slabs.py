"""Row-split runs of one domain: the rows are divided into slabs, one slab per
GPU (one process per GPU under torchrun, NCCL between them), or every slab
on one GPU in one process.

FloodCA's distributed run (src/mpi/halo.c:17-100, src/mpi/main_mpi.c:
113-160) gives each rank a block of a 2-D process grid with one ghost cell
on each side, owned cells [r0, r1) x [c0, c1) of FcaGrid
(src/common/fca_types.h:103-104), and per step exchanges the ghosts of h
before the fluxes and of the limiter s before the update
(src/common/model.c:359-360,507-508), with dt min-reduced over the ranks
(model.c:143-144) and the volumes sum-reduced at the end (model.c:627-629).

Here a slab is whole rows, and it carries three halo rows of each
neighbour's depth (FCAB_SLAB_HALO) in the padding rows of its session. The
step kernel recomputes the halo rows' faces, limiter and new depth itself,
as it does at every segment edge inside one GPU, so a step needs one
exchange of depth rows (after the step) and one max-reduction of the
velocity maximum (before the next dt is fixed), and no exchange of s. The
results equal a single-domain run bit for bit: the dt sequence is the same
because the velocity maximum is exact, and every cell sees the same
neighbours.
"""
from __future__ import annotations

import argparse
import contextlib
import ctypes as C
import json
import time
from dataclasses import dataclass
from types import SimpleNamespace

import numpy as np
import torch

from .lib import check
from .sim import Domain, RunParams, Session, _ptr, effective_rday

HALO = 3        # FCAB_SLAB_HALO


@dataclass(frozen=True)
class SlabSpec:
    """Own rows [r0, r1) of the domain and the halo rows above / below."""
    r0: int
    r1: int
    hn: int
    hs: int

    @property
    def rows(self) -> int:
        return self.r1 - self.r0


def slab_specs(nrows: int, parts: int) -> list[SlabSpec]:
    """Contiguous row ranges of near-equal size, each at least HALO rows (a
    neighbour's halo is filled from them alone)."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    if parts > 1 and nrows < parts * HALO:
        raise ValueError(f"{nrows} rows cannot make {parts} slabs of >= {HALO} rows")
    bounds = [nrows * i // parts for i in range(parts + 1)]
    return [SlabSpec(bounds[i], bounds[i + 1], HALO if i > 0 else 0,
                     HALO if i < parts - 1 else 0) for i in range(parts)]


def slab_domain(dom: Domain, p: RunParams, spec: SlabSpec) -> tuple[Domain, RunParams]:
    """The rasters of rows [r0 - hn, r1 + hs) and the slab's run parameters:
    internal edges closed, the inflow cell indexed in the slab's rows (or
    none when it lies outside them)."""
    a, b = spec.r0 - spec.hn, spec.r1 + spec.hs
    cut = lambda x: None if x is None else np.ascontiguousarray(x[a:b])
    d = Domain(cut(dom.z), cut(dom.mask), cut(dom.n), cut(dom.C), cut(dom.Rday), cut(dom.h),
               dom.dx, cut(dom.hmax), cut(dom.tmax))
    nr, nc = dom.shape
    edges = (p.edges[0] if spec.r0 == 0 else 0, p.edges[1] if spec.r1 == nr else 0,
             p.edges[2], p.edges[3])
    cell = -1
    if p.inflow_cell >= 0:
        r, c = divmod(int(p.inflow_cell), nc)
        if a <= r < b:
            cell = (r - a) * nc + c
    return d, p.with_(edges=edges, inflow_cell=cell)


class _DevWords:
    """A device address exposed to torch as a 1-element int64 tensor."""

    def __init__(self, ptr: int):
        self.__cuda_array_interface__ = {"shape": (1,), "typestr": "<i8",
                                         "data": (int(ptr), False), "version": 3,
                                         "stream": None}


class Slab(Session):
    """The session of one slab: own rows plus halo rows of its neighbours.
    `vmax` is a device view (int64) of the session's pending velocity
    maximum, valid while the slab is open."""

    def __init__(self, dom: Domain, p: RunParams, spec: SlabSpec, precision: str = "f32",
                 math: str = "exact", cols_per_lane: int = 0, seg_rows: int = 0, stream=None):
        d, q = slab_domain(dom, p, spec)
        self.spec = spec
        row_in = p.inflow_cell // dom.shape[1]
        self.owns_inflow = p.inflow_cell >= 0 and spec.r0 <= row_in < spec.r1
        self.dom = d.astype(np.float64 if precision == "f64" else np.float32)
        self._create(SimpleNamespace(shape=(spec.rows, dom.shape[1]), dx=dom.dx), q, precision,
                     math, cols_per_lane, seg_rows, stream)
        check(self.L.fcab_sim_set_slab(self.h, spec.hn, spec.hs), "fcab_sim_set_slab")
        d = self.dom
        R = effective_rday(d, q, self.dtype)
        check(self.L.fcab_sim_upload(self.h, _ptr(d.z), _ptr(d.h), _ptr(d.n), _ptr(d.C), _ptr(R),
                                     _ptr(d.mask), _ptr(d.hmax), _ptr(d.tmax)), "fcab_sim_upload")
        ptr = C.c_void_p()
        check(self.L.fcab_sim_slab_vmax(self.h, C.byref(ptr)), "fcab_sim_slab_vmax")
        self.vmax = torch.as_tensor(_DevWords(ptr.value), device="cuda")
        self.nc = dom.shape[1]
        self.torch_dtype = torch.float64 if precision == "f64" else torch.float32

    def step(self) -> None:
        check(self.L.fcab_sim_slab_step(self.h), "fcab_sim_slab_step")

    def finalize(self) -> None:
        check(self.L.fcab_sim_slab_finalize(self.h), "fcab_sim_slab_finalize")

    def vfull(self) -> None:
        check(self.L.fcab_sim_slab_vfull(self.h), "fcab_sim_slab_vfull")

    def rows_get(self, row0: int, buf: torch.Tensor) -> None:
        check(self.L.fcab_sim_rows_get(self.h, row0, buf.shape[0], C.c_void_p(buf.data_ptr())),
              "fcab_sim_rows_get")

    def rows_put(self, row0: int, buf: torch.Tensor) -> None:
        check(self.L.fcab_sim_rows_put(self.h, row0, buf.shape[0], C.c_void_p(buf.data_ptr())),
              "fcab_sim_rows_put")

    def rows_buffer(self, n: int) -> torch.Tensor:
        return torch.empty((n, self.nc), dtype=self.torch_dtype, device="cuda")


# ---------------------------------------------------------------------------
# Communication: every slab in this process, or one slab per rank.

class LocalSlabs:
    """Every slab on this GPU and one stream: the velocity maximum is reduced
    with a device max over the slabs, halo rows are copied device to
    device."""

    def __init__(self, slabs: list[Slab]):
        self.slabs = slabs
        self.bufs = [(s.rows_buffer(HALO), s.rows_buffer(HALO)) for s in slabs]

    def reduce_max(self) -> None:
        if len(self.slabs) == 1:
            return
        m = torch.stack([s.vmax for s in self.slabs]).amax(0)
        for s in self.slabs:
            s.vmax.copy_(m)

    def exchange(self) -> None:
        for i in range(len(self.slabs) - 1):
            a, b = self.slabs[i], self.slabs[i + 1]
            up, dn = self.bufs[i]
            a.rows_get(a.spec.rows - b.spec.hn, dn[:b.spec.hn])   # a's last rows: b's north halo
            b.rows_get(0, up[:a.spec.hs])                           # b's first rows: a's south halo
            b.rows_put(-b.spec.hn, dn[:b.spec.hn])
            a.rows_put(a.spec.rows, up[:a.spec.hs])


class RankSlab:
    """One slab per rank of a torch.distributed group: NCCL on device
    tensors, or (staged) gloo through host copies."""

    def __init__(self, slab: Slab, rank: int, world: int, staged: bool = False, group=None):
        self.slabs = [slab]
        self.rank, self.world, self.staged, self.group = rank, world, staged, group
        s = slab.spec
        self.send_n, self.recv_n = slab.rows_buffer(HALO), slab.rows_buffer(HALO)
        self.send_s, self.recv_s = slab.rows_buffer(HALO), slab.rows_buffer(HALO)
        self.has_n, self.has_s = s.hn > 0, s.hs > 0

    def reduce_max(self) -> None:
        import torch.distributed as dist
        v = self.slabs[0].vmax
        if self.staged:
            h = v.cpu()
            dist.all_reduce(h, op=dist.ReduceOp.MAX, group=self.group)
            v.copy_(h)
        else:
            dist.all_reduce(v, op=dist.ReduceOp.MAX, group=self.group)

    def exchange(self) -> None:
        import torch.distributed as dist
        s = self.slabs[0]
        # own first / last HALO rows go to the neighbours' halos
        if self.has_n:
            s.rows_get(0, self.send_n)
        if self.has_s:
            s.rows_get(s.spec.rows - HALO, self.send_s)
        pairs = []
        if self.has_n:
            pairs += [(self.send_n, self.recv_n, self.rank - 1)]
        if self.has_s:
            pairs += [(self.send_s, self.recv_s, self.rank + 1)]
        if not pairs:
            return
        if self.staged:
            host = [(a.cpu(), torch.empty(b.shape, dtype=b.dtype), peer) for a, b, peer in pairs]
            ops = []
            for a, b, peer in host:
                ops += [dist.P2POp(dist.isend, a, peer, self.group),
                        dist.P2POp(dist.irecv, b, peer, self.group)]
            for r in dist.batch_isend_irecv(ops):
                r.wait()
            for (a, b, _), (_, hb, _) in zip(pairs, host):
                b.copy_(hb)
        else:
            ops = []
            for a, b, peer in pairs:
                ops += [dist.P2POp(dist.isend, a, peer, self.group),
                        dist.P2POp(dist.irecv, b, peer, self.group)]
            for r in dist.batch_isend_irecv(ops):
                r.wait()
        if self.has_n:
            s.rows_put(-HALO, self.recv_n)
        if self.has_s:
            s.rows_put(s.spec.rows, self.recv_s)


def settle_dt(comm) -> None:
    """Fixes the pending dt on every slab: reduce the velocity maximum, let
    every slab decide; if the decision was deferred (the seed-pruned maximum
    fell below its seed, alike on every slab), the full velocity pass and a
    second reduction decide it (otherwise those do nothing)."""
    slabs = comm.slabs
    comm.reduce_max()
    for s in slabs:
        s.finalize()
    if hasattr(slabs[0], "vfull"):
        for s in slabs:
            s.vfull()
        comm.reduce_max()
        for s in slabs:
            s.finalize()


def run_slabs(comm, check_every: int = 32, max_iters: int | None = None) -> int:
    """Steps every slab to the end of the run. Each iteration fixes the
    pending dt from the reduced velocity maximum, takes one step and refills
    the halos; a finished slab's kernels do nothing, and every slab finishes
    at the same step. Returns the iterations taken."""
    slabs = comm.slabs
    st = slabs[0].stream()
    it = 0
    with (torch.cuda.stream(torch.cuda.ExternalStream(st)) if st else contextlib.nullcontext()):
        while max_iters is None or it < max_iters:
            for _ in range(check_every):
                settle_dt(comm)
                for s in slabs:
                    s.step()
                comm.exchange()
                it += 1
            if slabs[0].poll().done:
                break
    return it


def merge_stats(stats: list[dict], owns_inflow: list[bool]) -> dict:
    """Whole-domain figures from the slabs' own: volumes and counters sum
    over slabs; time, step and dt are the same on every slab; the inflow
    volume is counted once, by the slab that owns the inflow cell."""
    out = dict(stats[0])
    for k in ("V", "V0", "V_rain", "clamp_err", "V_sea", "V_bnd", "cap_active", "cap_total"):
        out[k] = sum(s[k] for s in stats)
    out["V_in"] = sum(s["V_in"] for s, o in zip(stats, owns_inflow) if o)
    den = max(out["V_rain"] + out["V_in"] + out["V0"], 1e-30)
    out["E_mass"] = abs(out["V"] + out["V_sea"] + out["V_bnd"] - out["V_rain"] - out["V_in"]
                        - out["V0"] - out["clamp_err"]) / den
    return out


def run_split_local(dom: Domain, p: RunParams, parts: int, **kw) -> dict:
    """Runs the domain as `parts` slabs on this GPU; returns h, hmax, tmax of
    the whole domain and the merged stats."""
    st = torch.cuda.Stream()
    slabs = [Slab(dom, p, spec, stream=C.c_void_p(st.cuda_stream), **kw)
             for spec in slab_specs(dom.shape[0], parts)]
    try:
        run_slabs(LocalSlabs(slabs))
        outs = [s.download() for s in slabs]
        stats = merge_stats([s.stats() for s in slabs], [s.owns_inflow for s in slabs])
    finally:
        for s in slabs:
            s.close()
    h, hmax, tmax = (np.concatenate([o[i] for o in outs]) for i in range(3))
    return {"h": h, "hmax": hmax, "tmax": tmax, **stats}


# ---------------------------------------------------------------------------

def main(argv=None) -> int:
    """Times a row-split run of the config-2 terrain: every slab on this GPU
    (--parts), or one slab per rank under torchrun (NCCL)."""
    import os

    from .profile_step import warm_config2
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=4096)
    ap.add_argument("--parts", type=int, default=2, help="slabs on this GPU (no torchrun)")
    ap.add_argument("--steps", type=int, default=400)
    args = ap.parse_args(argv)
    dom, p = warm_config2(args.size)
    p = p.with_(steps=args.steps, T_sim=30 * 86400.0)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    land = int((dom.mask == 0).sum())
    if world > 1:
        import torch.distributed as dist
        rank = int(os.environ["RANK"])
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", rank)))
        dist.init_process_group("nccl", device_id=torch.device("cuda", torch.cuda.current_device()))
        spec = slab_specs(dom.shape[0], world)[rank]
        slab = Slab(dom, p, spec)
        comm = RankSlab(slab, rank, world)
        parts = world
    else:
        st = torch.cuda.Stream()
        slabs = [Slab(dom, p, spec, stream=C.c_void_p(st.cuda_stream))
                 for spec in slab_specs(dom.shape[0], args.parts)]
        comm = LocalSlabs(slabs)
        parts = args.parts
    stream = torch.cuda.ExternalStream(comm.slabs[0].stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0.record(stream)
    n = run_slabs(comm, check_every=args.steps + 1)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t)
    steps = comm.slabs[0].stats()["step"]
    if int(os.environ.get("RANK", "0")) == 0:
        print(json.dumps({"workload": f"config-2 terrain {args.size}^2, row-split",
                          "slabs": parts, "ranks": world, "steps": steps, "iterations": n,
                          "ms": round(ms, 2), "wall_s": round(time.perf_counter() - t0, 2),
                          "gcells": round(land * steps / ms / 1e6, 2)}))
    for s in comm.slabs:
        s.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
