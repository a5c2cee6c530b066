"""ctypes mirrors of the C-ABI structs.

The Fca* structs repeat the layout of FloodCA's src/common/fca_types.h:34-159
(the CUDA backend's ABI, which callers fill and this library reads); the
Fcab* structs mirror include/floodca_b200.h. `real` is float or double
depending on the library build, so the Fca* classes are made per width by
fca_types(real).
"""
from __future__ import annotations

import ctypes as C
from functools import lru_cache

FCA_LAND, FCA_SEA, FCA_WALL = 0, 1, 2
FCA_BND_OPEN, FCA_BND_CLOSED = 0, 1
FCA_HYETO_TRIANGLE, FCA_HYETO_UNIFORM = 0, 1
FCA_MAX_FORCE_DAYS = 64

FCAB_PREC_F32, FCAB_PREC_F32_ALL, FCAB_PREC_F64 = 0, 1, 2
FCAB_MATH_EXACT, FCAB_MATH_FAST = 0, 1


class FcaTypes:
    """Namespace holding the Fca* ctypes classes for one `real` width."""

    def __init__(self, real):
        self.real = real
        rp = C.POINTER(real)

        class FcaPhys(C.Structure):
            _fields_ = [(n, real) for n in ("dx", "A", "g", "alpha", "tau_h", "tau_l", "z_sea",
                                            "dt_max", "dt_min", "S_bnd", "h_flood")] + \
                       [("U", C.c_int), ("K", C.c_int), ("boundary", C.c_int)]

        class FcaRunCfg(C.Structure):
            _fields_ = [
                ("phys", FcaPhys), ("T_sim", real), ("out_every", real),
                ("diag_every", C.c_int), ("progress_every", C.c_int), ("hyeto", C.c_int),
                ("D_h", real), ("phi", real), ("lambda_", real),
                ("steps", C.c_int), ("no_output", C.c_int), ("neigh", C.c_int),
                ("config_path", C.c_char * 512), ("grid_dir", C.c_char * 512),
                ("scenario", C.c_char * 128), ("scenario_file", C.c_char * 512),
                ("warmstart", C.c_char * 512), ("rain_file", C.c_char * 512),
                ("out_dir", C.c_char * 512), ("csv_path", C.c_char * 512),
                ("exp_id", C.c_char * 32), ("repeat", C.c_int), ("threads", C.c_int),
                ("ranks", C.c_int), ("gpus", C.c_int), ("block_x", C.c_int), ("block_y", C.c_int),
                ("halo_mode", C.c_char * 16), ("reduce_impl", C.c_char * 16),
                ("gpu_model", C.c_char * 64), ("backend", C.c_char * 32),
                ("forcing_csv", C.c_char * 512), ("n_force_days", C.c_int),
                ("force_files", (C.c_char * 768) * FCA_MAX_FORCE_DAYS),
            ]

        class FcaComm(C.Structure):
            # distributed-memory hooks; the function pointers are opaque here
            _fields_ = [("ctx", C.c_void_p), ("rank", C.c_int), ("halo", C.c_void_p),
                        ("min_real", C.c_void_p), ("sum_double", C.c_void_p),
                        ("load_rday", C.c_void_p)]

        class FcaGrid(C.Structure):
            _fields_ = [
                ("nrows", C.c_int), ("ncols", C.c_int), ("r0", C.c_int), ("r1", C.c_int),
                ("c0", C.c_int), ("c1", C.c_int), ("edge_n", C.c_int), ("edge_s", C.c_int),
                ("edge_w", C.c_int), ("edge_e", C.c_int), ("comm", C.c_void_p),
                ("dx", real), ("x0", real), ("y0", real),
                ("z", rp), ("h", rp), ("n", rp), ("C", rp), ("mask", C.POINTER(C.c_uint8)),
                ("Rday", rp), ("hmax", rp), ("tmax", rp), ("s", rp), ("out", rp),
                ("Qx", rp), ("Qy", rp), ("Qd1", rp), ("Qd2", rp), ("Qopen", rp),
            ]

        class FcaAcc(C.Structure):
            _fields_ = [
                ("V", C.c_double), ("V0", C.c_double), ("V_rain", C.c_double),
                ("V_sea", C.c_double), ("V_bnd", C.c_double), ("clamp_err", C.c_double),
                ("cap_active", C.c_long), ("cap_total", C.c_long), ("dt_min_hits", C.c_long),
                ("t", C.c_double), ("step", C.c_int), ("dt_base", real), ("force_day", C.c_int),
            ]

        class FcaTimers(C.Structure):
            _fields_ = [(n, C.c_double) for n in (
                "wall_total", "t_init", "t_flux", "t_limiter", "t_update", "t_dt", "t_io",
                "t_h2d", "t_d2h", "t_halo", "t_allreduce", "bytes_per_step")] + \
                [("active_cells", C.c_long)]

        self.FcaPhys, self.FcaRunCfg, self.FcaGrid = FcaPhys, FcaRunCfg, FcaGrid
        self.FcaComm = FcaComm
        self.FcaAcc, self.FcaTimers = FcaAcc, FcaTimers

    def offsets(self) -> dict[str, int]:
        """sizeof/offsetof table in the format of oracle/abi_probe.c."""
        out: dict[str, int] = {"sizeof(real)": C.sizeof(self.real)}
        names = {"lambda_": "lambda"}
        for cls in (self.FcaPhys, self.FcaRunCfg, self.FcaComm, self.FcaGrid, self.FcaAcc,
                    self.FcaTimers):
            out[f"sizeof({cls.__name__})"] = C.sizeof(cls)
            for f in cls._fields_:
                out[f"{cls.__name__}.{names.get(f[0], f[0])}"] = getattr(cls, f[0]).offset
        return out


@lru_cache(maxsize=2)
def fca_types(real=C.c_float) -> FcaTypes:
    return FcaTypes(real)


class FcabConfig(C.Structure):
    _fields_ = [
        ("nrows", C.c_int), ("ncols", C.c_int), ("precision", C.c_int), ("math", C.c_int),
        ("K", C.c_int), ("U", C.c_int), ("boundary", C.c_int),
        ("edge_n", C.c_int), ("edge_s", C.c_int), ("edge_w", C.c_int), ("edge_e", C.c_int),
        ("hyeto", C.c_int), ("max_steps", C.c_int),
        ("dx", C.c_double), ("g", C.c_double), ("alpha", C.c_double), ("tau_h", C.c_double),
        ("tau_l", C.c_double), ("z_sea", C.c_double), ("dt_max", C.c_double),
        ("dt_min", C.c_double), ("S_bnd", C.c_double),
        ("T_sim", C.c_double), ("out_every", C.c_double), ("D_h", C.c_double), ("phi", C.c_double),
        ("rain_end", C.c_double), ("inflow_cell", C.c_longlong),
        ("inflow_peak", C.c_double), ("inflow_t_peak", C.c_double), ("inflow_t_end", C.c_double),
        ("cols_per_lane", C.c_int), ("seg_rows", C.c_int),
    ]


class FcabStats(C.Structure):
    _fields_ = [
        ("t", C.c_double), ("dt_base", C.c_double), ("step", C.c_int), ("done", C.c_int),
        ("V", C.c_double), ("V0", C.c_double), ("V_rain", C.c_double), ("V_sea", C.c_double),
        ("V_bnd", C.c_double), ("clamp_err", C.c_double), ("V_in", C.c_double),
        ("cap_active", C.c_longlong), ("cap_total", C.c_longlong), ("dt_min_hits", C.c_longlong),
        ("E_mass", C.c_double), ("dt_full_passes", C.c_longlong),
    ]

    def as_dict(self) -> dict:
        return {f[0]: getattr(self, f[0]) for f in self._fields_}


class FcabPoll(C.Structure):
    _fields_ = [("t", C.c_double), ("dt_base", C.c_double), ("step", C.c_int),
                ("done", C.c_int), ("pause", C.c_int), ("force_day", C.c_int)]


class FcabInfo(C.Structure):
    _fields_ = [("cols_per_lane", C.c_int), ("grid", C.c_int), ("warps", C.c_int),
                ("ctas_per_sm", C.c_int), ("rain_field", C.c_int), ("land_only", C.c_int),
                ("land_cells", C.c_longlong), ("faces_per_step", C.c_longlong),
                ("pitch", C.c_longlong), ("tma_rows", C.c_int)]


class FcabBatchInfo(C.Structure):
    _fields_ = [("members", C.c_int), ("cols_per_lane", C.c_int), ("seg_rows", C.c_int),
                ("grid", C.c_int), ("total_units", C.c_int), ("launches", C.c_longlong),
                ("windows", C.c_longlong), ("graph_replays", C.c_longlong)]
