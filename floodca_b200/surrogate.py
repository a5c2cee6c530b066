"""Surrogate-screened flood ensembles (config 5: 10,000 members of 256 x 256).

Members are 256 x 256 grids of the config-4 generator (own terrain, Manning
n x lognormal(0, 0.3), uniform rain of 20-150 mm/h for 0.5-4 h, 8 h
simulated, open south edge). The CA (the batched WCA step) gives each
member's peak depth; the U-Net of floodca_b200/unet.py learns
(relief, n, rain intensity, rain duration) -> peak depth from 2000 CA runs
(200 more for validation). Screening: MC-dropout passes of the surrogate
over every member; members whose predicted area above 0.3 m exceeds the
area threshold, or whose predictive spread exceeds 0.1 m, are re-run in the
CA; the others keep the surrogate's mean prediction.

Reported: members/hour of the screened ensemble against the plain CA
ensemble (every member in the batched CA), and the screened ensemble's
accuracy against the CA: RMSE of peak depth and CSI at 0.1 m,
CSI = hits / (hits + false alarms + misses) (FloodCA
prep/floodca_prep/validation_metrics.py:98-106). Setup (terrain and input
generation, session upload) is outside every timed region.

    python -m floodca_b200.surrogate [--members 10000] [--train 2000] [--out res.json]
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time
from pathlib import Path

import numpy as np

from .ensemble import Batch, Member, member_session, terrain_torch

SIDE = 256
DEPTH_SCALE = 0.1          # target transform t = log1p(hmax / DEPTH_SCALE)


def members(n: int, seed: int, side: int = SIDE, T_sim: float = 8 * 3600.0) -> list[Member]:
    rng = np.random.default_rng(seed)
    return [Member(side=side, seed=int(seed * 1000003 + i), n_scale=float(rng.lognormal(0, 0.3)),
                   rain_mm_h=float(rng.uniform(20.0, 150.0)),
                   rain_h=float(rng.uniform(0.5, 4.0)), T_sim=T_sim) for i in range(n)]


def inputs(ms: list[Member], device="cuda"):
    """fp32 [N, H, W, 4]: relief (z - mean) / 10, n / 0.1, rain / 150 mm/h,
    duration / 4 h."""
    import torch
    out = torch.empty((len(ms), ms[0].side, ms[0].side, 4), dtype=torch.float32, device=device)
    for i, m in enumerate(ms):
        z, n = terrain_torch(m.side, m.seed, n_scale=m.n_scale, device=device)
        out[i, :, :, 0] = (z - z.mean()) / 10.0
        out[i, :, :, 1] = n / 0.1
        out[i, :, :, 2] = m.rain_mm_h / 150.0
        out[i, :, :, 3] = m.rain_h / 4.0
    return out


def run_ca(ms: list[Member], chunk: int = 2500, tuning=None) -> tuple:
    """Peak depth of every member from the batched CA (device fp32
    [N, H, W]) and the CA's timed seconds (sessions set up untimed)."""
    import torch
    from .ensemble import DEFAULT_TUNING, seg_for
    tuning = tuning or DEFAULT_TUNING
    H = ms[0].side
    hmax = torch.empty((len(ms), H, H), dtype=torch.float32, device="cuda")
    wall = 0.0
    for c0 in range(0, len(ms), chunk):
        part = ms[c0:c0 + chunk]
        sessions = [member_session(m) for m in part]
        torch.cuda.synchronize()
        b = Batch(sessions, tuning["cols_per_lane"], 0, [seg_for(m.side, tuning) for m in part])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b.run(window=0.0, graph_steps=32)
        torch.cuda.synchronize()
        wall += time.perf_counter() - t0
        b.close()
        for i, s in enumerate(sessions):
            _, hm, _ = s.download()
            hmax[c0 + i] = torch.from_numpy(hm)
            s.close()
    return hmax, wall


def to_target(hmax):
    import torch
    return torch.log1p(hmax.clamp_min(0.0) / DEPTH_SCALE)


def from_target(t):
    import torch
    return DEPTH_SCALE * torch.expm1(t.clamp_min(0.0))


def train(model, X, Y, Xv=None, Yv=None, epochs: int = 30, batch: int = 32, lr: float = 2e-3,
          seed: int = 0, log=None) -> dict:
    """Adam on the mean squared error of the transformed peak depth, cosine
    learning-rate decay, dropout active."""
    import torch
    rng = np.random.default_rng(seed)
    n = X.shape[0]
    steps = epochs * (n // batch)
    hist = []
    t0 = time.perf_counter()
    k = 0
    for ep in range(epochs):
        perm = rng.permutation(n)
        tot = torch.zeros(1, device="cuda")
        for j in range(n // batch):
            idx = torch.as_tensor(perm[j * batch:(j + 1) * batch], device="cuda")
            xb, yb = X[idx].contiguous(), Y[idx].contiguous()
            model.forward(xb, dropout_seed=int(rng.integers(1, 1 << 30)))
            model.backward(yb)
            cur = lr * 0.5 * (1 + math.cos(math.pi * k / max(1, steps)))
            model.adam(lr=cur)
            tot += model.loss_sum
            k += 1
        torch.cuda.synchronize()
        rec = {"epoch": ep + 1, "train_mse": float(tot) / (n // batch * batch * X.shape[1] * X.shape[2]),
               "s": time.perf_counter() - t0}
        if Xv is not None and ((ep + 1) % 5 == 0 or ep + 1 == epochs):
            pv = predict_mean(model, Xv)
            rec["val_rmse_m"] = float(((pv - from_target(Yv)) ** 2).mean().sqrt())
        hist.append(rec)
        if log:
            log(rec)
    if model.device_error():
        raise RuntimeError("surrogate kernels reported a device error")
    return {"steps": k, "seconds": time.perf_counter() - t0, "history": hist}


def predict_mean(model, X, batch: int = 64):
    """Deterministic prediction (no dropout) of peak depth, metres."""
    import torch
    out = torch.empty(X.shape[:3], dtype=torch.float32, device="cuda")
    for i in range(0, X.shape[0], batch):
        out[i:i + batch] = from_target(model.forward(X[i:i + batch].contiguous()))
    return out


def predict_mc(model, X, passes: int = 8, batch: int = 64, seed: int = 1):
    """MC-dropout mean and standard deviation of peak depth (metres)."""
    import torch
    N = X.shape[0]
    mean = torch.zeros(X.shape[:3], dtype=torch.float32, device="cuda")
    sq = torch.zeros_like(mean)
    for i in range(0, N, batch):
        xb = X[i:i + batch].contiguous()
        for p in range(passes):
            d = from_target(model.forward(xb, dropout_seed=seed * 1000 + p + 1))
            mean[i:i + batch] += d
            sq[i:i + batch] += d * d
    mean /= passes
    var = (sq / passes - mean * mean).clamp_min(0.0)
    return mean, var.sqrt()


def metrics(pred, truth, thr: float = 0.1) -> dict:
    """RMSE of peak depth (m) and CSI at thr over all cells of all members."""
    import torch
    e = (pred - truth).double()
    p, t = pred > thr, truth > thr
    hits = int((p & t).sum())
    fa = int((p & ~t).sum())
    miss = int((~p & t).sum())
    return {"rmse_m": float(e.pow(2).mean().sqrt()), "csi_0p1": hits / max(1, hits + fa + miss),
            "hits": hits, "false_alarms": fa, "misses": miss}


def screen(model, X, passes: int = 8, area_thr_cells: int | None = None,
           area_quantile: float = 0.9, spread_thr: float = 0.1, batch: int = 64) -> dict:
    """Surrogate pass over every member: per member the predicted area above
    0.3 m (cells) and the spread (mean over the predicted wet cells, > 0.1
    m, of the MC-dropout standard deviation). Returns the flags of members
    to re-run, the mean prediction and the timing (set-up excluded: one
    untimed forward pass at the screening batch size first, as the CA
    ensembles' session set-up is outside their timing)."""
    import torch
    model.forward(X[:batch].contiguous(), dropout_seed=1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    mean, std = predict_mc(model, X, passes, batch=batch)
    area = (mean > 0.3).flatten(1).sum(1)
    wet = (mean > 0.1).flatten(1)
    spread = (std.flatten(1) * wet).sum(1) / wet.sum(1).clamp_min(1)
    torch.cuda.synchronize()
    t_sur = time.perf_counter() - t0
    if area_thr_cells is None:
        area_thr_cells = int(torch.quantile(area.float(), area_quantile))
    rerun = (area > area_thr_cells) | (spread > spread_thr)
    return {"mean": mean, "rerun": rerun.cpu().numpy(), "area_thr_cells": area_thr_cells,
            "t_surrogate_s": t_sur, "spread": spread.cpu().numpy(), "area": area.cpu().numpy()}


def screened_vs_plain(model, ms: list[Member], passes: int = 8, batch: int = 64) -> dict:
    """The plain CA ensemble of ms and the surrogate-screened one: timings,
    members/hour and the screened ensemble's accuracy against the CA."""
    import torch
    Yall, t_ca = run_ca(ms)
    Xall = inputs(ms)
    sc = screen(model, Xall, passes=passes, batch=batch)
    rer = np.nonzero(sc["rerun"])[0]
    Yre, t_re = run_ca([ms[i] for i in rer]) if len(rer) else (None, 0.0)
    final = sc["mean"].clone()
    if len(rer):
        final[torch.as_tensor(rer, device="cuda")] = Yre
    n = len(ms)
    return {"plain_s": t_ca, "plain_members_per_hour": n / t_ca * 3600.0,
            "surrogate_s": sc["t_surrogate_s"], "rerun_members": int(len(rer)), "rerun_s": t_re,
            "screened_members_per_hour": n / (sc["t_surrogate_s"] + t_re) * 3600.0,
            "accuracy": metrics(final, Yall), "surrogate_only": metrics(sc["mean"], Yall),
            "area_thr_cells": sc["area_thr_cells"]}


def layer_bench(N: int = 64, steps: int = 10, warmup: int = 3, train_batch: int = 32) -> dict:
    """Device time of MC-dropout forward passes (N images) and of training
    steps (forward, backward, Adam) on random inputs, CUDA events on the
    current stream."""
    import torch
    from .unet import UNet
    model = UNet(seed=0)
    model.prep()
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    X = torch.randn((N, SIDE, SIDE, 4), device="cuda", generator=g)
    Y = torch.rand((train_batch, SIDE, SIDE), device="cuda", generator=g)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for i in range(warmup):
        model.forward(X, dropout_seed=i + 1)
    torch.cuda.synchronize()
    e0.record()
    for i in range(steps):
        model.forward(X, dropout_seed=i + 100)
    e1.record()
    e1.synchronize()
    t_fwd = e0.elapsed_time(e1) / steps / 1e3
    Xt = X[:train_batch].contiguous()
    for i in range(warmup):
        model.forward(Xt, dropout_seed=i + 1)
        model.backward(Y)
        model.adam(lr=1e-4)
    torch.cuda.synchronize()
    e0.record()
    for i in range(steps):
        model.forward(Xt, dropout_seed=i + 100)
        model.backward(Y)
        model.adam(lr=1e-4)
    e1.record()
    e1.synchronize()
    t_tr = e0.elapsed_time(e1) / steps / 1e3
    if model.device_error():
        raise RuntimeError("surrogate kernels reported a device error")
    ff = model.flops_forward(N, SIDE, SIDE)
    ft = 3.0 * model.flops_forward(train_batch, SIDE, SIDE)
    return {"forward": {"images": N, "ms": t_fwd * 1e3, "tflops": ff / t_fwd / 1e12,
                        "images_per_s": N / t_fwd},
            "train_step": {"images": train_batch, "ms": t_tr * 1e3, "tflops": ft / t_tr / 1e12}}


def conv_bench(N: int, H: int, Cin: int, Cout: int, steps: int = 5, warmup: int = 2) -> dict:
    """Device time of one 3x3 convolution layer (forward) on N images of
    H x H, random bf16 inputs."""
    import torch
    from .lib import core
    from .unet import bordered
    L = core()
    x = bordered(N, H, H, Cin)
    x.view(N, H + 2, H + 2, Cin)[:, 1:-1, 1:-1].normal_()
    w = torch.randn((Cout, 9, Cin), device="cuda") / math.sqrt(9 * Cin)
    wb = torch.empty((Cout, 9, Cin), dtype=torch.bfloat16, device="cuda")
    wt = torch.empty((Cin, 9, Cout), dtype=torch.bfloat16, device="cuda")
    L.fcab_unet_prep_weights(_ptr(w), _ptr(wb), _ptr(wt), Cout, Cin, None)
    b = torch.zeros(Cout, device="cuda")
    y = bordered(N, H, H, Cout)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(warmup):
        L.fcab_unet_conv_fwd(_ptr(x), N, H, H, Cin, _ptr(wb), Cout, _ptr(b), 1, _ptr(y), None)
    e0.record()
    for _ in range(steps):
        L.fcab_unet_conv_fwd(_ptr(x), N, H, H, Cin, _ptr(wb), Cout, _ptr(b), 1, _ptr(y), None)
    e1.record()
    e1.synchronize()
    t = e0.elapsed_time(e1) / steps / 1e3
    flops = 2.0 * N * H * H * 9 * Cin * Cout
    return {"conv": [N, H, Cin, Cout], "ms": t * 1e3, "tflops": flops / t / 1e12,
            "error": L.fcab_unet_device_error()}


def _ptr(t):
    import ctypes as C
    return C.c_void_p(t.data_ptr())


def main(argv=None) -> int:
    import torch
    from .unet import UNet
    ap = argparse.ArgumentParser()
    ap.add_argument("--conv-bench", default="",
                    help="N,H,Cin,Cout: time one convolution layer only")
    ap.add_argument("--layer-bench", action="store_true",
                    help="time forward passes and training steps on random inputs only")
    ap.add_argument("--members", type=int, default=10000)
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--val", type=int, default=200)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--passes", type=int, default=8)
    ap.add_argument("--hours", type=float, default=8.0)
    ap.add_argument("--weights", default="", help="save the trained weights (.npz)")
    ap.add_argument("--out", default="")
    a = ap.parse_args(argv)
    if a.layer_bench:
        print(json.dumps(layer_bench()))
        return 0
    if a.conv_bench:
        N, H, ci, co = (int(v) for v in a.conv_bench.split(","))
        print(json.dumps(conv_bench(N, H, ci, co)))
        return 0
    T = a.hours * 3600.0
    log = lambda r: print(json.dumps(r), flush=True)
    # training data from the CA
    tr = members(a.train, seed=11, T_sim=T)
    va = members(a.val, seed=12, T_sim=T)
    Ytr, t_tr = run_ca(tr)
    Yva, _ = run_ca(va)
    Xtr, Xva = inputs(tr), inputs(va)
    log({"ca_training_runs": a.train + a.val, "ca_s": t_tr})
    model = UNet(seed=0)
    model.prep()
    fit = train(model, Xtr, to_target(Ytr), Xva, to_target(Yva), epochs=a.epochs, log=log)
    del Xtr, Ytr
    if a.weights:
        np.savez(a.weights, **model.state_dict())
    val = metrics(predict_mean(model, Xva), Yva)
    # the screening ensemble
    ms = members(a.members, seed=13, T_sim=T)
    Yall, t_ca = run_ca(ms)
    Xall = inputs(ms)
    sc = screen(model, Xall, passes=a.passes)
    rer = np.nonzero(sc["rerun"])[0]
    Yre, t_re = run_ca([ms[i] for i in rer]) if len(rer) else (None, 0.0)
    final = sc["mean"].clone()
    if len(rer):
        final[torch.as_tensor(rer, device="cuda")] = Yre
    flops = model.flops_forward(a.members, SIDE, SIDE) * a.passes
    res = {
        "workload": f"config 5: {a.members} members of {SIDE}x{SIDE}, {a.hours:g} h simulated; "
                    f"U-Net trained on {a.train} CA runs, validated on {a.val}",
        "training": {"steps": fit["steps"], "seconds": fit["seconds"],
                     "final": fit["history"][-1], "val": val},
        "plain_ca": {"seconds": t_ca, "members_per_hour": a.members / t_ca * 3600.0},
        "screened": {
            "surrogate_s": sc["t_surrogate_s"], "rerun_members": int(len(rer)),
            "rerun_ca_s": t_re, "seconds": sc["t_surrogate_s"] + t_re,
            "members_per_hour": a.members / (sc["t_surrogate_s"] + t_re) * 3600.0,
            "area_thr_cells": sc["area_thr_cells"], "passes": a.passes,
            "surrogate_tflops": flops / sc["t_surrogate_s"] / 1e12,
            "accuracy_vs_ca": metrics(final, Yall),
            "surrogate_only_accuracy": metrics(sc["mean"], Yall),
        },
    }
    res["speedup_members_per_hour"] = (res["screened"]["members_per_hour"] /
                                       res["plain_ca"]["members_per_hour"])
    txt = json.dumps(res, indent=1)
    if a.out:
        Path(a.out).write_text(txt + "\n")
    print(txt)
    return 0


if __name__ == "__main__":
    sys.exit(main())
