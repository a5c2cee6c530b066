"""A fixed workload of the step kernel for profilers (ncu): the warm 4096^2
config-2 grid of the benchmark (20 mm everywhere), `--steps` steps of one
session. Prints the session's launch shape; it makes no timing claim.

    python -m floodca_b200.profile_step [--size 4096] [--steps 24] [--math exact] [--cpl 0]
"""
from __future__ import annotations

import argparse
import json
import sys

import numpy as np

from . import synth
from .sim import Session


def warm_config2(n: int = 4096):
    """Config-2 terrain of side n with 20 mm of water everywhere (the
    benchmark's warm start)."""
    dom, p = synth.config2(n=n)
    dom = dom.copy()
    dom.h = np.full(dom.shape, 0.02, np.float32)
    dom.hmax = dom.h.copy()
    return dom, p


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=4096)
    ap.add_argument("--steps", type=int, default=24)
    ap.add_argument("--math", default="exact")
    ap.add_argument("--cpl", type=int, default=0)
    a = ap.parse_args(argv)
    dom, p = warm_config2(a.size)
    with Session(dom, p.with_(T_sim=30 * 86400.0), precision="f32", math=a.math,
                 cols_per_lane=a.cpl) as s:
        s.advance(a.steps)
        st = s.stats()
        print(json.dumps({"info": s.info(), "step": st["step"], "t": st["t"]}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
