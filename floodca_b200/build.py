"""Builds the floodca_b200 shared libraries in-tree for sm_100a.

Outputs (next to this file):
  libfloodca_b200_core.so  kernels + the fcab_* session API
  libfloodca_b200.so       drop-in fca_cuda_* ABI, float `real`
  libfloodca_b200_f64.so   drop-in fca_cuda_* ABI, double `real` (FCA_DOUBLE)

Run `python -m floodca_b200.build` (or `__graft_entry__.build()`). Objects
go to _build/ at the repository root. Sources are rebuilt only when newer
than their object. FCAB_NVCC_FLAGS adds nvcc flags (for example the launch
shape macro -DFCAB_PAIR_WARPS=12); changing it needs a clean _build/.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = ROOT / "_build"

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --fmad=false keeps a*b+c as two rounded operations, as the reference's
# parity build does on the host (-ffp-contract=off); explicit fmaf() calls
# in the kernels are unaffected. It does not stop ptxas from fusing a packed
# mul.rn.f32x2 into a following add.rn.f32x2 (nor does ptxas's own
# --fmad=false); the pair sweep forms such products with scalar mul.rn.
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "--fmad=false",
           "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", "-I", str(INCLUDE), "-I", str(CSRC),
           *os.environ.get("FCAB_NVCC_FLAGS", "").split()]

CORE_SRCS = ["wca_inst_f32.cu", "wca_inst_f32all.cu", "wca_inst_f64.cu", "wca_inst_batch.cu",
             "wca_sim.cu", "host_copy.cu", "mem_cache.cu", "wca_noalloc.cu", "wca_batch.cu", "unet_tc.cu"]


def _deps_newer(obj: Path, srcs: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(s.stat().st_mtime > t for s in srcs)


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [INCLUDE / "floodca_b200.h"]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def _compile(src: Path, obj: Path, extra: list[str]) -> Path:
    if _deps_newer(obj, [src] + _headers()):
        _run([NVCC, *ARCH, *NVFLAGS, *extra, "-c", str(src), "-o", str(obj)])
    return obj


# The step kernels launch the full velocity pass from the device (a tail
# launch, dynamic parallelism): their units are compiled as relocatable
# device code and the core library links the device runtime.
RDC_SRCS = {"wca_inst_f32.cu", "wca_inst_f32all.cu", "wca_inst_f64.cu"}


def build(verbose: bool = True, jobs: int | None = None) -> dict[str, Path]:
    """Compiles every CUDA/C++ source and links the three libraries."""
    BUILD.mkdir(exist_ok=True)
    jobs = jobs or min(8, os.cpu_count() or 4)
    tasks = [(CSRC / s, BUILD / (Path(s).stem + ".o"), ["-rdc=true"] if s in RDC_SRCS else [])
             for s in CORE_SRCS]
    tasks.append((CSRC / "abi_dropin.cpp", BUILD / "abi_dropin_f32.o", ["-x", "cu"]))
    tasks.append((CSRC / "abi_dropin.cpp", BUILD / "abi_dropin_f64.o", ["-x", "cu", "-DFCA_DOUBLE"]))
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda t: _compile(*t), tasks))
    core_objs, shim32, shim64 = objs[:len(CORE_SRCS)], objs[-2], objs[-1]

    out = {"core": PKG / "libfloodca_b200_core.so", "f32": PKG / "libfloodca_b200.so",
           "f64": PKG / "libfloodca_b200_f64.so"}
    link = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC"]
    if _deps_newer(out["core"], core_objs):
        _run([*link, *map(str, core_objs), "-lcudadevrt", "-o", str(out["core"])])
    for key, shim in (("f32", shim32), ("f64", shim64)):
        if _deps_newer(out[key], [shim, out["core"]]):
            _run([*link, str(shim), "-L", str(PKG), "-lfloodca_b200_core",
                  "-Xlinker", "-rpath=$ORIGIN", "-o", str(out[key])])
    if verbose:
        for k, p in out.items():
            print(f"built {k}: {p.relative_to(ROOT)}")
    return out


if __name__ == "__main__":
    build(verbose=True)
    sys.exit(0)
