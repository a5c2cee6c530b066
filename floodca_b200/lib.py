"""Loads the in-tree floodca_b200 shared libraries.

The product path is the CUDA code in these libraries; there is no CPU
fallback. If a library is missing this module raises immediately with the
build command.
"""
from __future__ import annotations

import ctypes as C
from functools import lru_cache
from pathlib import Path

from .abi import FcabBatchInfo, FcabConfig, FcabInfo, FcabPoll, FcabStats, fca_types

PKG = Path(__file__).resolve().parent
LIB_CORE = PKG / "libfloodca_b200_core.so"
LIB_F32 = PKG / "libfloodca_b200.so"
LIB_F64 = PKG / "libfloodca_b200_f64.so"


class LibraryMissing(ImportError):
    pass


def _load(path: Path) -> C.CDLL:
    if not path.exists():
        raise LibraryMissing(f"{path.name} is not built; run `python -m floodca_b200.build`")
    return C.CDLL(str(path))


_P = C.c_void_p
_I = C.c_int
_LL = C.c_longlong


@lru_cache(maxsize=1)
def core() -> C.CDLL:
    """The kernels and the fcab_* session API."""
    L = _load(LIB_CORE)
    sim_pp = C.POINTER(C.c_void_p)
    sig = {
        "fcab_config_defaults": (None, [C.POINTER(FcabConfig), C.c_int, C.c_int]),
        "fcab_sim_create": (C.c_int, [sim_pp, C.POINTER(FcabConfig), _P]),
        "fcab_sim_upload": (C.c_int, [_P] * 9),
        "fcab_sim_upload_device": (C.c_int, [_P] * 9),
        "fcab_sim_upload_state": (C.c_int, [_P] * 4),
        "fcab_sim_set_rain": (C.c_int, [_P, _P, _P]),
        "fcab_sim_set_config": (C.c_int, [_P, C.POINTER(FcabConfig)]),
        "fcab_sim_set_pause_every": (C.c_int, [_P, C.c_int, C.c_int]),
        "fcab_sim_advance": (C.c_int, [_P, C.c_int]),
        "fcab_sim_run": (C.c_int, [_P]),
        "fcab_sim_reset_time": (C.c_int, [_P, C.c_double, C.c_int, C.c_double, C.c_int]),
        "fcab_sim_poll": (C.c_int, [_P, C.POINTER(FcabPoll)]),
        "fcab_sim_resume": (C.c_int, [_P, C.c_int]),
        "fcab_sim_info": (C.c_int, [_P, C.POINTER(FcabInfo)]),
        "fcab_sim_stats": (C.c_int, [_P, C.POINTER(FcabStats)]),
        "fcab_sim_download": (C.c_int, [_P, _P, _P, _P]),
        "fcab_sim_layout": (C.c_int, [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P),
                                      C.POINTER(C.c_longlong), C.POINTER(C.c_int),
                                      C.POINTER(C.c_int)]),
        "fcab_sim_count_flooded": (C.c_int, [_P, C.c_int, C.POINTER(C.c_double), _P,
                                             C.POINTER(C.c_longlong), C.POINTER(C.c_double)]),
        "fcab_sim_launches": (C.c_longlong, [_P]),
        "fcab_sim_stream": (_P, [_P]),
        "fcab_release_cached_memory": (None, []),
        "fcab_sim_set_slab": (C.c_int, [_P, _I, _I]),
        "fcab_sim_slab_step": (C.c_int, [_P]),
        "fcab_sim_slab_vfull": (C.c_int, [_P]),
        "fcab_sim_slab_vmax": (C.c_int, [_P, C.POINTER(_P)]),
        "fcab_sim_slab_finalize": (C.c_int, [_P]),
        "fcab_sim_rows_get": (C.c_int, [_P, _I, _I, _P]),
        "fcab_sim_rows_put": (C.c_int, [_P, _I, _I, _P]),
        "fcab_sim_destroy": (None, [_P]),
        "fcab_math_probe": (C.c_int, [C.c_int, _P, _P, _P, C.c_longlong, C.c_float]),
        "fcab_batch_create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_int,
                                        C.c_int, C.c_int, C.POINTER(C.c_int), _P]),
        "fcab_batch_run": (C.c_int, [_P, C.c_double, C.c_int, C.c_int]),
        "fcab_batch_info": (C.c_int, [_P, C.POINTER(FcabBatchInfo)]),
        "fcab_batch_destroy": (None, [_P]),
        "fcab_run_noalloc": (C.c_int, [C.POINTER(FcabConfig), _P, _P, _P, _P, _P, _P, _P, _P,
                                       _P, C.POINTER(FcabStats)]),
        # surrogate layers
        "fcab_unet_conv_fwd": (C.c_int, [_P, _I, _I, _I, _I, _P, _I, _P, _I, _P, _P]),
        "fcab_unet_conv_dgrad": (C.c_int, [_P, _I, _I, _I, _I, _P, _I, _P, _P]),
        "fcab_unet_conv_wgrad": (C.c_int, [_P, _P, _I, _I, _I, _I, _I, _P, _P]),
        "fcab_unet_maxpool2": (C.c_int, [_P, _P, _P, _I, _I, _I, _I, _P]),
        "fcab_unet_maxpool2_bwd": (C.c_int, [_P, _P, _P, _I, _I, _I, _I, _P]),
        "fcab_unet_maxpool2_bwd_add": (C.c_int, [_P, _P, _P, _I, _I, _P, _I, _I, _I, _I, _P]),
        "fcab_unet_upcat": (C.c_int, [_P, _I, _P, _I, _P, _I, _I, _I, _P]),
        "fcab_unet_upcat_bwd": (C.c_int, [_P, _I, _I, _P, _I, _I, _I, _P]),
        "fcab_unet_upsample2": (C.c_int, [_P, _P, _I, _I, _I, _I, _P]),
        "fcab_unet_upsample2_bwd": (C.c_int, [_P, _P, _I, _I, _I, _I, _P]),
        "fcab_unet_concat": (C.c_int, [_P, _I, _P, _I, _P, _I, _I, _I, _I, _P]),
        "fcab_unet_add": (C.c_int, [_P, _P, _LL, _P]),
        "fcab_unet_relu_bwd": (C.c_int, [_P, _P, _LL, _P]),
        "fcab_unet_dropout": (C.c_int, [_P, _LL, C.c_float, C.c_uint32, _P]),
        "fcab_unet_bias_grad": (C.c_int, [_P, _LL, _I, _P, _P]),
        "fcab_unet_head_fwd": (C.c_int, [_P, _P, _P, _P, _I, _I, _I, _I, _P]),
        "fcab_unet_head_bwd": (C.c_int, [_P] * 8 + [_I, _I, _I, _I, _P]),
        "fcab_unet_prep_weights": (C.c_int, [_P, _P, _P, _I, _I, _P]),
        "fcab_unet_adam": (C.c_int, [_P, _P, _P, _P, _LL, C.c_float, C.c_float, C.c_float,
                                     C.c_float, _I, C.c_float, _P]),
        "fcab_unet_pack_input": (C.c_int, [_P, _I, _P, _I, _I, _I, _I, _P]),
        "fcab_unet_device_error": (C.c_int, []),
        "fcab_unet_wait_probe": (C.c_int, [_LL, _P]),
        "fcab_last_error": (C.c_char_p, []),
        "fcab_version": (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype, fn.argtypes = res, args
    return L


@lru_cache(maxsize=2)
def dropin(double: bool = False) -> C.CDLL:
    """The reference-facing fca_cuda_* ABI (float or double `real`)."""
    core()
    L = _load(LIB_F64 if double else LIB_F32)
    T = fca_types(C.c_double if double else C.c_float)
    L.fca_cuda_run.restype = C.c_int
    L.fca_cuda_run.argtypes = [C.POINTER(T.FcaGrid), C.POINTER(T.FcaRunCfg),
                               C.POINTER(T.FcaAcc), C.POINTER(T.FcaTimers)]
    L.fca_cuda_device_name.restype = None
    L.fca_cuda_device_name.argtypes = [C.c_char_p, C.c_size_t]
    L.fca_cuda_select_device.restype = C.c_int
    L.fca_cuda_select_device.argtypes = [C.c_int]
    L.fca_cuda_ens_open.restype = _P
    L.fca_cuda_ens_open.argtypes = [C.POINTER(T.FcaGrid), C.POINTER(T.FcaRunCfg), C.c_int,
                                    C.POINTER(C.c_double)]
    L.fca_cuda_ens_run.restype = C.c_int
    L.fca_cuda_ens_run.argtypes = [_P, C.POINTER(T.FcaGrid), C.POINTER(T.FcaRunCfg),
                                   C.POINTER(T.FcaAcc), C.POINTER(T.FcaTimers),
                                   C.POINTER(C.c_long), C.POINTER(C.c_double), _P, _P, C.c_int]
    L.fca_cuda_ens_counts.restype = C.c_int
    L.fca_cuda_ens_counts.argtypes = [_P, C.POINTER(C.c_uint16)]
    L.fca_cuda_ens_close.restype = None
    L.fca_cuda_ens_close.argtypes = [_P]
    return L


def last_error() -> str:
    return core().fcab_last_error().decode()


class FcabError(RuntimeError):
    pass


def check(rc: int, what: str) -> None:
    if rc != 0:
        raise FcabError(f"{what} failed ({rc}): {last_error()}")
