"""Comparison of a CUDA run's result with the compiled reference core
(oracle/_ref/libfcaref_*.so, the reference's src/common built with its parity
flags) on the same domain and parameters: FP32 bit for bit; FP64 depths
within 1e-12 m and times within 1e-9 s (the device's and glibc's double cube
roots may differ in the last bit); the volumes within 1e-9 relative.

Test helper only (imported by the GPU tests)."""
import numpy as np
import pytest

from oracle import refcore


def reference(d, p, kind="f32"):
    if not refcore.available(kind):
        pytest.skip("reference core not built")
    return refcore.run(d, p, kind=kind)


def check(r, ref, kind="f32", volumes=("V", "V_rain", "V_sea", "V_bnd", "V_in", "clamp_err")):
    """r: a result dict (h, hmax, tmax, step, t and the volumes)."""
    assert r["step"] == ref["step"], (r["step"], ref["step"])
    if kind == "f32":
        assert r["t"] == ref["t"], (r["t"], ref["t"])
    else:
        assert r["t"] == pytest.approx(ref["t"], abs=1e-9)
    for k in ("h", "hmax", "tmax"):
        a = np.asarray(r[k])
        if kind == "f32":
            assert np.array_equal(a, ref[k]), (k, float(np.abs(a - ref[k]).max()))
        else:
            tol = 1e-9 if k == "tmax" else 1e-12
            assert np.abs(a.astype(np.float64) - ref[k]).max() <= tol, k
    for k in volumes:
        assert r[k] == pytest.approx(ref[k], rel=1e-9, abs=1e-6), k
    if "cap_active" in r:
        assert r["cap_active"] == ref["cap_active"]


def check_reference(r, d, p, kind="f32", **kw):
    """Runs the reference core on (d, p) and compares r with it."""
    ref = reference(d, p, kind)
    check(r, ref, kind, **kw)
    return ref
