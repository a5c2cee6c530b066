"""Command line: runs a grid directory on the GPU through a session, with the
options of the reference's CLIs (FloodCA src/common/cli.c:19-95,
src/common/config.c:56-212: `--key value` or `--key=value`, an optional
`--config` file of `key = value` lines) plus this project's extensions, and
writes hmax / h_final in the reference's output format.

    python -m floodca_b200 --grid DIR [--steps N | --tsim T] [--neigh 4|8] [--U N]
        [--boundary open|closed] [--hyeto triangle|uniform] [--D_h D] [--phi P]
        [--rain FILE --lambda L] [--warmstart FILE] [--out_every S] [--out DIR]
        [--no-output] [--g --alpha --tau_h --tau_l --z_sea --dt_max --dt_min --S_bnd]
      extensions: [--edges NSWE, e.g. 0100: open south only] [--rain_end S]
        [--inflow_cell R,C --inflow_peak Q --inflow_t_peak T --inflow_t_end T]
        [--precision f32|f32all|f64] [--math exact|fast]

Forcing days (`--forcing`) run through the reference's own CLI linked against
the drop-in library, which handles the daily rain reloads.
"""
from __future__ import annotations

import sys
from dataclasses import dataclass, field

import numpy as np

from .sim import Domain, RunParams

# RunParams field of each reference key (config.c:56-130 set_kv), with its type
_KEYS = {
    "g": ("g", float), "alpha": ("alpha", float), "tau_h": ("tau_h", float),
    "tau_l": ("tau_l", float), "z_sea": ("z_sea", float), "dt_max": ("dt_max", float),
    "dt_min": ("dt_min", float), "S_bnd": ("S_bnd", float), "U": ("U", int),
    "K": ("K", int), "neigh": ("K", int), "T_sim": ("T_sim", float), "tsim": ("T_sim", float),
    "out_every": ("out_every", float), "D_h": ("D_h", float), "phi": ("phi", float),
    "lambda": ("lambda_", float), "steps": ("steps", int),
    # extensions
    "rain_end": ("rain_end", float), "inflow_peak": ("inflow_peak", float),
    "inflow_t_peak": ("inflow_t_peak", float), "inflow_t_end": ("inflow_t_end", float),
}


@dataclass
class Options:
    grid: str = ""
    out: str = ""
    no_output: bool = False
    rain: str = ""
    warmstart: str = ""
    precision: str = "f32"
    math: str = "exact"
    inflow_rc: tuple | None = None
    params: dict = field(default_factory=dict)


class UsageError(ValueError):
    pass


def _set(o: Options, k: str, v: str) -> None:
    if k in _KEYS:
        name, typ = _KEYS[k]
        o.params[name] = typ(v)
    elif k == "boundary":
        o.params["boundary"] = "closed" if v == "closed" else "open"
    elif k == "hyeto":
        o.params["hyeto"] = "uniform" if v == "uniform" else "triangle"
    elif k == "edges":
        if len(v) != 4 or set(v) - {"0", "1"}:
            raise UsageError("--edges takes four 0/1 flags in the order N S W E")
        o.params["edges"] = tuple(int(ch) for ch in v)
    elif k == "inflow_cell":
        r, c = (int(x) for x in v.split(","))
        o.inflow_rc = (r, c)
    elif k in ("grid", "out", "rain", "warmstart"):
        setattr(o, k, v)
    elif k == "precision":
        if v not in ("f32", "f32all", "f64"):
            raise UsageError("--precision is f32, f32all or f64")
        o.precision = v
    elif k == "math":
        if v not in ("exact", "fast"):
            raise UsageError("--math is exact or fast")
        o.math = v
    elif k in ("forcing", "forcing_csv"):
        raise UsageError("forcing days: run the reference's CLI against the drop-in library")
    # other reference keys (threads, block, csv, exp, reduce, ...) do not
    # change a GPU session's results and are accepted silently


def parse(argv: list[str]) -> Options:
    """Options from the command line, in the reference's grammar."""
    o = Options()
    i = 0
    while i < len(argv):
        a = argv[i]
        if a in ("-h", "--help"):
            raise UsageError(__doc__)
        if not a.startswith("--"):
            i += 1
            continue
        if a == "--no-output":
            o.no_output = True
            i += 1
            continue
        if "=" in a:
            k, v = a[2:].split("=", 1)
        elif i + 1 < len(argv):
            k, v = a[2:], argv[i + 1]
            i += 1
        else:
            k, v = a[2:], None
        i += 1
        if v is None:
            continue
        if k == "config":
            for ln in open(v).read().splitlines():
                ln = ln.split("#", 1)[0].strip()
                if "=" in ln:
                    kk, vv = (s.strip() for s in ln.split("=", 1))
                    _set(o, kk, vv)
        else:
            _set(o, k, v)
    if not o.grid:
        raise UsageError("--grid DIR is required")
    return o


def inputs(o: Options) -> tuple[Domain, RunParams]:
    """The grid directory with the rain file and warm start applied, as the
    reference's CLIs load them (main_cuda.c:39-55, grid.c:239-268), and the
    run parameters."""
    from .synth import read_grid_dir
    dom = read_grid_dir(o.grid)
    kw = dict(o.params)
    lam = kw.pop("lambda_", 1.0)
    n = dom.shape[0] * dom.shape[1]
    if o.rain:
        # fca_grid_load_rday + lambda: Rday = file * lambda (float32 raster)
        dom.Rday = np.fromfile(o.rain, np.float32, n).reshape(dom.shape)
        kw["lambda_"] = lam
    if o.warmstart:
        dom.h = np.fromfile(o.warmstart, np.float32, n).reshape(dom.shape)
    dom.hmax = dom.h.copy()
    if o.inflow_rc is not None:
        r, c = o.inflow_rc
        if not (0 <= r < dom.shape[0] and 0 <= c < dom.shape[1]):
            raise UsageError("--inflow_cell outside the grid")
        kw["inflow_cell"] = r * dom.shape[1] + c
    return dom, RunParams(**kw)


def main(argv: list[str] | None = None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    try:
        o = parse(argv)
        dom, p = inputs(o)
    except UsageError as e:
        if e.args and e.args[0] == __doc__:
            print(__doc__)
            return 0                # the reference's CLIs exit 0 after --help
        print(str(e), file=sys.stderr)
        return 1
    from .lib import FcabError, core
    from .sim import Session
    print(f"floodca backend=b200 dx={dom.dx:g} K={p.K} U={p.U} boundary={p.boundary} "
          f"steps={p.steps} T_sim={p.T_sim:g} precision={o.precision}", flush=True)
    try:
        with Session(dom, p, precision=o.precision, math=o.math) as s:
            s.run()
            st = s.stats()
            print(f"done backend=b200 steps={st['step']} t={st['t']:.6g} "
                  f"E_mass={st['E_mass']:.3e} V={st['V']:.6g} "
                  f"{core().fcab_version().decode()}", flush=True)
            if o.out and not o.no_output:
                s.write_outputs(o.out)
    except FcabError as e:
        print(f"floodca_b200: {e}", file=sys.stderr)
        return 1
    return 0
