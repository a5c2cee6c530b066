"""ctypes wrapper of oracle/conv_ref.c, the CPU reference of the surrogate's
3x3 convolutions (test infrastructure: used by tests only).

Arrays are float32 NHWC [N, H, W, C]; weights [Cout, 9, Cin]."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

_LIB = Path(__file__).resolve().parent / "libconv_ref.so"
_P = C.c_void_p
_I = C.c_int


def _lib():
    if not _LIB.exists():
        raise ImportError(f"{_LIB.name} is not built; run `make -C oracle`")
    L = C.CDLL(str(_LIB))
    L.conv_ref_fwd.argtypes = [_P, _I, _I, _I, _I, _P, _I, _P, _I, _P]
    L.conv_ref_dgrad.argtypes = [_P, _I, _I, _I, _I, _P, _I, _P]
    L.conv_ref_wgrad.argtypes = [_P, _P, _I, _I, _I, _I, _I, _P]
    for f in (L.conv_ref_fwd, L.conv_ref_dgrad, L.conv_ref_wgrad):
        f.restype = None
    return L


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


def fwd(x, w, bias=None, relu=False):
    x, w = _f32(x), _f32(w)
    N, H, W, Cin = x.shape
    Cout = w.shape[0]
    y = np.empty((N, H, W, Cout), np.float32)
    b = None if bias is None else _f32(bias)
    _lib().conv_ref_fwd(_ptr(x), N, H, W, Cin, _ptr(w), Cout, _ptr(b), int(relu), _ptr(y))
    return y


def dgrad(dy, w):
    dy, w = _f32(dy), _f32(w)
    N, H, W, Cout = dy.shape
    Cin = w.shape[2]
    dx = np.empty((N, H, W, Cin), np.float32)
    _lib().conv_ref_dgrad(_ptr(dy), N, H, W, Cout, _ptr(w), Cin, _ptr(dx))
    return dx


def wgrad(dy, x):
    dy, x = _f32(dy), _f32(x)
    N, H, W, Cout = dy.shape
    Cin = x.shape[3]
    dw = np.empty((Cout, 9, Cin), np.float32)
    _lib().conv_ref_wgrad(_ptr(dy), _ptr(x), N, H, W, Cin, Cout, _ptr(dw))
    return dw
