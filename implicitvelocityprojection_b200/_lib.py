"""ctypes binding of `libivp.so` (the C ABI in include/ivp.h).

The library is loaded from this package directory.  There is no fallback: if
it is missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

from . import build as _build

OK = 0
NOT_SPD = 1
NOT_CONVERGED = 2
NBR_OVERFLOW = 3
BAD_ARG = 4
CUDA_ERROR = 5
TIMEOUT = 6
NOT_BOUND = 7
DEVICE_CHECK = 8


class SceneDesc(ctypes.Structure):
    _fields_ = [
        ("particle_offset", ctypes.c_int32),
        ("n_particles", ctypes.c_int32),
        ("n_dynamic", ctypes.c_int32),
        ("particle_radius", ctypes.c_float),
        ("domain_size", ctypes.c_float * 3),
        ("dt", ctypes.c_float),
        ("gravity", ctypes.c_float * 3),
        ("omega", ctypes.c_float),
        ("tol_pcg", ctypes.c_double),
        ("density_error_tol", ctypes.c_double),
        ("max_outer_iters", ctypes.c_int32),
        ("max_iteration_pcg", ctypes.c_int32),
        ("fixed_outer_iters", ctypes.c_int32),
        ("cache_size", ctypes.c_int32),
        ("viscosity_coeff", ctypes.c_float),
        ("viscosity_method", ctypes.c_int32),
        ("surface_tension_method", ctypes.c_int32),
        ("surface_tension_coeff", ctypes.c_float),
        ("pressure_solver", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 1),
    ]


class Options(ctypes.Structure):
    _fields_ = [
        ("lanes_per_particle", ctypes.c_int32),
        ("particles_per_block", ctypes.c_int32),
        ("list_stride", ctypes.c_int32),
        ("max_hist", ctypes.c_int32),
        ("use_graphs", ctypes.c_int32),
        ("persistent", ctypes.c_int32),
        ("row_format", ctypes.c_int32),
        ("build_kernel", ctypes.c_int32),
    ]


class Particles(ctypes.Structure):
    _fields_ = [
        ("x", ctypes.c_void_p),
        ("v", ctypes.c_void_p),
        ("m", ctypes.c_void_p),
        ("density0", ctypes.c_void_p),
        ("is_dynamic", ctypes.c_void_p),
        ("material", ctypes.c_void_p),
        ("density", ctypes.c_void_p),
        ("kdiag", ctypes.c_void_p),
        ("divergence", ctypes.c_void_p),
        ("n_total", ctypes.c_int32),
    ]


class SolveStats(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int32),
        ("outer_iters", ctypes.c_int32),
        ("n_density_errors", ctypes.c_int32),
        ("overflow_particles", ctypes.c_int32),
        ("final_density_error", ctypes.c_double),
        ("last_density_error", ctypes.c_double),
        ("total_pcg_iters", ctypes.c_int32),
        ("solves", ctypes.c_int32),
        ("failed_solves", ctypes.c_int32),
        ("last_failure", ctypes.c_int32),
        ("sum_outer_iters", ctypes.c_int64),
        ("sum_pcg_iters", ctypes.c_int64),
        ("max_final_density_error", ctypes.c_double),
        ("neighbour_pairs", ctypes.c_int64),
        ("sum_visc_iters", ctypes.c_int64),
        ("sum_st_iters", ctypes.c_int64),
        ("last_pap", ctypes.c_double),
        ("last_cg_iter", ctypes.c_int32),
        ("fixup_entries", ctypes.c_int32),
    ]


# kernel ids of ivp_profile_step (include/ivp.h)
KERNEL_NAMES = ["gravity", "solve_begin", "pack", "rhs", "cg_a", "cg_b", "solve_end", "divergence", "advect",
                "keys", "scan_local", "scan_add", "place", "order", "nbr_build", "static_out", "visc", "ip_solve",
                "surface_tension", "prj"]
K_COUNT = 24
NOALLOC_MAX_PARTICLES = 65536
NOALLOC_MAX_CELLS = 262144


# every exported symbol of include/ivp.h with its ctypes signature
_P = ctypes.c_void_p
_I = ctypes.c_int32
SIGNATURES = {
    "ivp_default_options": (None, [ctypes.POINTER(Options)]),
    "ivp_workspace_bytes": (_I, [ctypes.POINTER(SceneDesc), _I, ctypes.POINTER(Options), ctypes.POINTER(ctypes.c_size_t)]),
    "ivp_resolve_options": (_I, [ctypes.POINTER(SceneDesc), _I, ctypes.POINTER(Options), ctypes.POINTER(Options)]),
    "ivp_engine_create": (_I, [ctypes.POINTER(SceneDesc), _I, ctypes.POINTER(Options), _P, ctypes.c_size_t, _P,
                               ctypes.POINTER(_P)]),
    "ivp_engine_destroy": (_I, [_P]),
    "ivp_update_scene": (_I, [_P, _I, ctypes.POINTER(SceneDesc), _P]),
    "ivp_engine_bind": (_I, [_P, ctypes.POINTER(Particles)]),
    "ivp_neighbour_build": (_I, [_P, _P]),
    "ivp_compute_density": (_I, [_P, _P]),
    "ivp_compute_aii": (_I, [_P, _P]),
    "ivp_ip_solve": (_I, [_P, _P]),
    "ivp_viscosity_solve": (_I, [_P, _P]),
    "ivp_surface_tension_solve": (_I, [_P, _P]),
    "ivp_prj_solve": (_I, [_P, _P]),
    "ivp_apply_gravity": (_I, [_P, _P]),
    "ivp_advect": (_I, [_P, _P]),
    "ivp_step": (_I, [_P, _I, _P]),
    "ivp_step_io": (_I, [_P, _P, _P, _P, _P, ctypes.c_int64, ctypes.c_int64, _P]),
    "ivp_reset_counters": (_I, [_P, _P]),
    "ivp_profile_step": (_I, [_P, _I, _P, _P, _P]),
    "ivp_read_stats": (_I, [_P, _I, _P, ctypes.POINTER(SolveStats)]),
    "ivp_read_history": (_I, [_P, _I, _P, _P, _P, _I, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "ivp_read_solve": (_I, [_P, _I, _P, ctypes.POINTER(SolveStats), _P, _P, _I, ctypes.POINTER(_I),
                            ctypes.POINTER(_I)]),
    "ivp_export_neighbours": (_I, [_P, _I, _P, _P, _I, _P]),
    "ivp_set_wait_limit": (_I, [_P, ctypes.c_int64]),
    "ivp_prepare": (_I, [_P]),
    "ivp_read_stats_all": (_I, [_P, _P, ctypes.POINTER(SolveStats)]),
    "ivp_density_aii_noalloc": (_I, [_P, _P, _P, _I, ctypes.c_float, _P, _I, _P, _P, _P]),
    "ivp_status_string": (ctypes.c_char_p, [_I]),
    "ivp_last_error": (ctypes.c_char_p, []),
}

_lib = None


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Loads libivp.so (building it with nvcc if it is absent or stale)."""
    global _lib
    if _lib is not None:
        return _lib
    if build_if_missing:
        _build.build()
    if not os.path.exists(_build.LIB):
        raise RuntimeError(f"libivp.so not found at {_build.LIB}; run python -m implicitvelocityprojection_b200.build")
    L = ctypes.CDLL(_build.LIB)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


class IVPError(RuntimeError):
    def __init__(self, status: int, where: str):
        L = load(False)
        msg = L.ivp_status_string(status).decode()
        detail = L.ivp_last_error().decode()
        super().__init__(f"{where}: {msg}" + (f" ({detail})" if detail and status == CUDA_ERROR else ""))
        self.status = status


def check(status: int, where: str) -> None:
    if status != OK:
        raise IVPError(int(status), where)
