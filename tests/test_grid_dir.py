"""The synthetic generator's grid directories (floodca_b200.synth
write_grid_dir) in the reference's format: the reference's own loader
(fca_grid_load_dir, src/common/grid.c:162-237, compiled in oracle/_ref)
reads back exactly the rasters that were written; CPU only."""
import ctypes as C

import numpy as np
import pytest

from floodca_b200 import abi, synth
from oracle import refcore

pytestmark = pytest.mark.skipif(not refcore.available("f32"), reason="reference core not built")


def _load_with_reference(path, kind):
    L = refcore.lib(kind)
    T = abi.fca_types(C.c_double if kind == "f64" else C.c_float)
    L.fca_grid_load_dir.restype = C.c_int
    L.fca_grid_load_dir.argtypes = [C.POINTER(T.FcaGrid), C.c_char_p]
    L.fca_grid_free.restype = None
    L.fca_grid_free.argtypes = [C.POINTER(T.FcaGrid)]
    g = T.FcaGrid()
    assert L.fca_grid_load_dir(C.byref(g), str(path).encode()) == 0
    try:
        nr, nc = g.nrows, g.ncols
        f = lambda ptr: np.ctypeslib.as_array(ptr, (nr, nc)).copy()
        out = dict(nrows=nr, ncols=nc, dx=float(g.dx), z=f(g.z), n=f(g.n), C=f(g.C),
                   Rday=f(g.Rday), h=f(g.h), hmax=f(g.hmax),
                   mask=np.ctypeslib.as_array(g.mask, (nr, nc)).copy(),
                   edges=(g.edge_n, g.edge_s, g.edge_w, g.edge_e))
    finally:
        L.fca_grid_free(C.byref(g))
    return out


@pytest.mark.parametrize("kind", ["f32", "f64"])
def test_reference_loader_reads_written_grid(tmp_path, kind):
    d = synth.make_terrain(synth.TerrainSpec(37, 53, seed=4, dx=45.0))
    rng = np.random.default_rng(0)
    d.h = rng.uniform(0, 0.3, d.shape).astype(np.float32)
    d.Rday = rng.uniform(0, 0.2, d.shape).astype(np.float32)
    d.C = rng.uniform(0.2, 1, d.shape).astype(np.float32)
    d.mask[0, :5] = abi.FCA_SEA
    d.mask[10, 10:20] = abi.FCA_WALL
    synth.write_grid_dir(d, tmp_path / "g")
    r = _load_with_reference(tmp_path / "g", kind)
    assert (r["nrows"], r["ncols"], r["dx"]) == (37, 53, 45.0)
    for k in ("z", "n", "C", "Rday", "h"):
        assert np.array_equal(r[k], getattr(d, k).astype(r[k].dtype)), k
    assert np.array_equal(r["hmax"], r["h"]) and np.array_equal(r["mask"], d.mask)
    back = synth.read_grid_dir(tmp_path / "g")
    for k in ("z", "n", "C", "Rday", "h", "mask"):
        assert np.array_equal(getattr(back, k), getattr(d, k)), k


def test_reference_loader_defaults_for_missing_rasters(tmp_path):
    d = synth.make_terrain(synth.TerrainSpec(8, 9, seed=1))
    synth.write_grid_dir(d, tmp_path / "g")
    for name in ("n", "C", "Rday", "h"):
        (tmp_path / "g" / f"{name}.bin").unlink()
    r = _load_with_reference(tmp_path / "g", "f32")
    back = synth.read_grid_dir(tmp_path / "g")
    for k, v in (("n", 0.03), ("C", 0.0), ("Rday", 0.0), ("h", 0.0)):
        assert np.all(r[k] == np.float32(v)) and np.array_equal(getattr(back, k), r[k]), k


@pytest.mark.parametrize("kind", ["f32", "f64"])
def test_output_field_matches_reference_writer(tmp_path, kind):
    """synth.write_field writes the same raster bytes and header fields as
    the reference's fca_grid_write_field (src/common/grid.c:271-306)."""
    import json
    L = refcore.lib(kind)
    dbl = kind == "f64"
    T = abi.fca_types(C.c_double if dbl else C.c_float)
    L.fca_grid_write_field.restype = C.c_int
    L.fca_grid_write_field.argtypes = [C.POINTER(T.FcaGrid), C.c_char_p, C.c_char_p,
                                       C.POINTER(T.real)]
    rng = np.random.default_rng(2)
    arr = rng.uniform(0, 3, (11, 7)).astype(np.float64 if dbl else np.float32)
    g = T.FcaGrid()
    g.nrows, g.ncols, g.dx, g.x0, g.y0 = 11, 7, 90.0, 500000.0, 1450000.0
    ref_dir, my_dir = tmp_path / "ref", tmp_path / "mine"
    ref_dir.mkdir()
    assert L.fca_grid_write_field(C.byref(g), str(ref_dir).encode(), b"hmax",
                                  arr.ctypes.data_as(C.POINTER(T.real))) == 0
    synth.write_field(my_dir, "hmax", arr, 90.0, 500000.0, 1450000.0)
    assert (my_dir / "hmax.bin").read_bytes() == (ref_dir / "hmax.bin").read_bytes()
    a = json.loads((ref_dir / "hmax.json").read_text())
    b = json.loads((my_dir / "hmax.json").read_text())
    a.pop("created"), b.pop("created")
    assert a == b
    assert np.array_equal(synth.read_field(my_dir, "hmax", arr.shape), arr)
