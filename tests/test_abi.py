"""The drop-in ABI: struct layouts match the reference's fca_types.h, and
the libraries export every entry point include/floodca_b200.h declares."""
import ctypes as C
import json
import re
import subprocess

import pytest

from conftest import GOLDEN, ROOT
from floodca_b200 import abi, lib


@pytest.mark.parametrize("kind,real", [("f32", C.c_float), ("f64", C.c_double)])
def test_ctypes_layout_matches_reference(kind, real):
    ref = json.loads((GOLDEN / "abi_layout.json").read_text())[kind]
    mine = abi.fca_types(real).offsets()
    assert {k: mine.get(k) for k in ref} == ref


@pytest.mark.parametrize("kind,flag", [("f32", []), ("f64", ["-DFCA_DOUBLE"])])
def test_header_layout_matches_reference(tmp_path, kind, flag):
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=gnu11", "-DPROBE_OWN_HEADER", *flag, "-I", str(ROOT / "include"),
                    "-o", str(exe), str(ROOT / "oracle" / "abi_probe.c")], check=True)
    mine = json.loads(subprocess.check_output([str(exe)]))
    ref = json.loads((GOLDEN / "abi_layout.json").read_text())[kind]
    assert mine == ref


def declared_symbols():
    text = (ROOT / "include" / "floodca_b200.h").read_text()
    return sorted(set(re.findall(r"^FCAB_API [^(]*?\b(fcab?_\w+)\(", text, re.M)))


def exported(path):
    out = subprocess.check_output(["nm", "-D", "--defined-only", str(path)], text=True)
    return {ln.split()[-1] for ln in out.splitlines() if " T " in ln}


def test_libraries_export_every_declared_symbol():
    syms = declared_symbols()
    assert "fca_cuda_run" in syms and "fcab_sim_create" in syms
    core = exported(lib.LIB_CORE)
    for shim in (lib.LIB_F32, lib.LIB_F64):
        ex = exported(shim) | core
        missing = [s for s in syms if s not in ex]
        assert not missing, f"{shim.name} lacks {missing}"


def test_libraries_load_without_gpu():
    L = lib.core()
    assert b"sm_100a" in L.fcab_version()
    for dbl in (False, True):
        D = lib.dropin(dbl)
        assert hasattr(D, "fca_cuda_run")


def test_config_defaults_match_reference():
    c = abi.FcabConfig()
    lib.core().fcab_config_defaults(C.byref(c), 10, 20)
    assert (c.nrows, c.ncols, c.K, c.U, c.boundary) == (10, 20, 4, 1, abi.FCA_BND_OPEN)
    assert (c.dx, c.g, c.alpha, c.tau_h, c.tau_l) == (30.0, 9.81, 0.5, 1e-3, 1e-5)
    assert (c.dt_max, c.dt_min, c.S_bnd, c.T_sim, c.D_h, c.phi) == (60.0, 0.01, 0.001, 86400.0, 24.0, 0.5)
