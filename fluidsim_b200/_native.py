"""ctypes binding of libfluidcuda.so (the C ABI declared in include/fluidcuda.h).

The library is built in place by fluidsim_b200/build.py. There is no fallback: if the library
is missing or cannot be loaded, importing the product raises, so no caller ever runs a silent
CPU substitute.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(HERE, "libfluidcuda.so")

FC_OK = 0
STATUS_NAMES = {
    0: "ok", 1: "invalid argument", 2: "lifecycle", 3: "cuda", 4: "out of memory",
    5: "non-finite", 6: "breakdown", 7: "unsupported", 8: "timeout",
}

PRECISION = {"fp32": 0, "fp64": 1, "mixed": 2}
PRECONDITIONER = {"diagonal": 0, "multigrid": 1}
TRANSPORT = {"semi_lagrangian": 0, "plic": 1}
AIR_MODEL = {"gas": 0, "dirichlet": 1}
SOLVE_STATUS = {0: "running", 1: "converged", 2: "iteration_limit", 3: "stalled", 4: "no_work", 5: "breakdown"}


class FcResult(C.Structure):
    """Mirror of fc_result (fluid::FluidProjectionResult plus solver measurements)."""
    _fields_ = [
        ("iterations", C.c_int),
        ("max_divergence", C.c_double),
        ("converged", C.c_int),
        ("physical_steps", C.c_int),
        ("transport_steps", C.c_int),
        ("relaxed", C.c_int),
        ("max_volume_error", C.c_double),
        ("rms_volume_error", C.c_double),
        ("viscosity_iterations", C.c_int),
        ("precision_limited", C.c_int),
        ("solve_status", C.c_int),
        ("residual_max", C.c_double),
        ("residual_l2", C.c_double),
        ("rhs_l2", C.c_double),
        ("divergence_excess", C.c_double),
        ("divergence_l2", C.c_double),
        ("restarts", C.c_int),
        ("kernels", C.c_int),
        ("refreshes", C.c_int),
    ]


class FcTimings(C.Structure):
    _fields_ = [(name, C.c_double) for name in
                ("transport_ms", "viscosity_ms", "forces_ms", "pressure_ms", "selection_ms", "regrid_ms")]


class FcSimDesc(C.Structure):
    """Mirror of fc_sim_desc: one simulation submitted to the serving loop."""
    _fields_ = [
        ("width", C.c_int), ("height", C.c_int), ("cell_size", C.c_double), ("precision", C.c_int),
        ("liquid_count", C.c_int), ("liquid_densities", C.c_void_p),
        ("gas_count", C.c_int), ("gas_densities", C.c_void_p),
        ("gravity_y", C.c_double), ("surface_tension", C.c_double),
        ("solid", C.c_void_p),
        ("liquid_fraction", C.c_void_p), ("u", C.c_void_p), ("v", C.c_void_p), ("pressure", C.c_void_p),
        ("liquid_mass", C.c_void_p), ("gas_mass", C.c_void_p),
        ("steps", C.c_int), ("dt", C.c_double), ("max_iterations", C.c_int), ("divergence_tolerance", C.c_double),
    ]


class FcSimStatus(C.Structure):
    _fields_ = [
        ("state", C.c_int), ("error", C.c_int), ("steps_done", C.c_int), ("physical_steps", C.c_int),
        ("iterations", C.c_longlong), ("converged", C.c_int), ("max_divergence", C.c_double),
        ("queued_ms", C.c_double), ("run_ms", C.c_double), ("device_bytes", C.c_size_t),
    ]


class FcServerStats(C.Structure):
    _fields_ = [
        ("ticks", C.c_longlong), ("steps", C.c_longlong), ("physical_steps", C.c_longlong),
        ("cell_steps", C.c_double), ("busy_ms", C.c_double),
        ("step_p50_ms", C.c_double), ("step_p99_ms", C.c_double), ("step_max_ms", C.c_double),
        ("peak_active", C.c_int), ("peak_bytes", C.c_size_t), ("batch_rebuilds", C.c_longlong),
    ]


_dp = C.POINTER(C.c_double)
_dpp = C.POINTER(_dp)
_vp = C.c_void_p
_int = C.c_int
_dbl = C.c_double

# name -> (restype, argtypes)
SIGNATURES = {
    "fc_abi_version": (_int, []),
    "fc_last_error": (C.c_char_p, []),
    "fc_status_string": (C.c_char_p, [_int]),
    "fc_kernel_launches": (C.c_longlong, []),
    "fc_set_launch_mode": (_int, [_int]),
    "fc_create": (_int, [_int, _int, _dbl, _int, C.POINTER(_vp)]),
    "fc_destroy": (_int, [_vp]),
    "fc_get_geometry": (_int, [_vp, C.POINTER(_int), C.POINTER(_int), _dp]),
    "fc_get_origin": (_int, [_vp, _dp, _dp]),
    "fc_set_origin": (_int, [_vp, _dbl, _dbl]),
    "fc_get_precision": (_int, [_vp, C.POINTER(_int)]),
    "fc_configure_materials": (_int, [_vp, _int, _dp, _dp, _int, _dp, _dp]),
    "fc_get_gravity": (_int, [_vp, _dp]),
    "fc_set_gravity": (_int, [_vp, _dbl]),
    "fc_set_preconditioner": (_int, [_vp, _int]),
    "fc_set_obstacles": (_int, [_vp, C.POINTER(C.c_uint8)]),
    "fc_upload": (_int, [_vp, _dp, _dp, _dp, _dp, _dpp, _dpp]),
    "fc_download": (_int, [_vp, _dp, _dp, _dp, _dp, _dpp, _dpp]),
    "fc_copy_state": (_int, [_vp, _vp]),
    "fc_project": (_int, [_vp, _dbl, _int, _dbl, C.POINTER(FcResult)]),
    "fc_project_relative": (_int, [_vp, _dbl, _int, _dbl, _dbl, C.POINTER(FcResult)]),
    "fc_step": (_int, [_vp, _dbl, _int, _dbl, C.POINTER(FcResult), C.POINTER(FcTimings)]),
    "fc_advect": (_int, [_vp, _dbl]),
    "fc_set_transport": (_int, [_vp, _int]),
    "fc_get_transport": (_int, [_vp, C.POINTER(_int)]),
    "fc_autotune": (_int, [_vp, _int, C.POINTER(_int), _dp]),
    "fc_batch_autotune": (_int, [_vp, _int, C.POINTER(_int), _dp]),
    "fc_set_tail_cells": (_int, [_vp, _int]),
    "fc_apply_viscosity": (_int, [_vp, _dbl, _dbl, _int, C.POINTER(_int), _dp]),
    "fc_set_component_viscosity": (_int, [_vp, _int, _int, _dbl]),
    "fc_grid_device_bytes": (_int, [_int, _int, _int, _int, _int, C.POINTER(C.c_size_t)]),
    "fc_get_device_bytes": (_int, [_vp, C.POINTER(C.c_size_t)]),
    "fc_server_create": (_int, [C.c_size_t, _int, C.POINTER(_vp)]),
    "fc_server_create_classes": (_int, [C.c_size_t, _int, _int, C.POINTER(C.c_longlong), C.POINTER(_vp)]),
    "fc_server_class_count": (_int, [_vp, C.POINTER(_int)]),
    "fc_server_get_class_stats": (_int, [_vp, _int, C.POINTER(FcServerStats), C.POINTER(C.c_longlong)]),
    "fc_server_destroy": (_int, [_vp]),
    "fc_server_submit": (_int, [_vp, C.POINTER(FcSimDesc), C.POINTER(C.c_longlong)]),
    "fc_server_status": (_int, [_vp, C.c_longlong, C.POINTER(FcSimStatus)]),
    "fc_server_wait": (_int, [_vp, C.c_longlong, _dbl, C.POINTER(FcSimStatus)]),
    "fc_server_download": (_int, [_vp, C.c_longlong, _vp, _vp, _vp, _vp, _vp, _vp]),
    "fc_server_release": (_int, [_vp, C.c_longlong]),
    "fc_server_error": (_int, [_vp, C.c_longlong, C.c_char_p, C.c_size_t]),
    "fc_server_get_stats": (_int, [_vp, C.POINTER(FcServerStats)]),
    "fc_server_step_latencies": (_int, [_vp, _vp, C.c_size_t, C.POINTER(C.c_size_t)]),
    "fc_get_surface_tension": (_int, [_vp, _dp]),
    "fc_set_surface_tension": (_int, [_vp, _dbl]),
    "fc_capillary_step_limit": (_int, [_vp, _dp]),
    "fc_apply_surface_tension": (_int, [_vp, _dbl]),
    "fc_surface_curvature": (_int, [_vp, _vp, _vp]),
    "fc_sample_velocity": (_int, [_vp, _int, _vp, _vp]),
    "fc_apply_gravity": (_int, [_vp, _dbl]),
    "fc_max_divergence": (_int, [_vp, _dp]),
    "fc_classify": (_int, [_vp, C.POINTER(C.c_uint8)]),
    "fc_set_air_model": (_int, [_vp, _int]),
    "fc_get_air_model": (_int, [_vp, C.POINTER(_int)]),
    "fc_extend_air_velocity": (_int, [_vp]),
    "fc_advance_substep": (_int, [_vp, _dbl, C.POINTER(_int)]),
    "fc_set_stream_priority": (_int, [_vp, _int]),
    "fc_download_coefficients": (_int, [_vp, _dp, _dp, _dp]),
    "fc_apply_preconditioner": (_int, [_vp, _dp, _dbl, _dp]),
    "fc_time_kernel": (_int, [_vp, _int, _int, _dp]),
    "fc_divergence_noalloc": (_int, [_vp, _vp, _int, _int, _dbl, _int, _vp, _vp]),
    "fc_velocity_pointers": (_int, [_vp, C.POINTER(_vp), C.POINTER(_vp)]),
    "fc_get_stream": (_int, [_vp, C.POINTER(_vp)]),
    "fc_synchronize": (_int, [_vp]),
    "fc_save_checkpoint": (_int, [_vp, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t), _vp, C.c_size_t,
                                  C.POINTER(C.c_size_t)]),
    "fc_load_checkpoint": (_int, [_vp, C.c_char_p, _vp, C.c_size_t]),
    "fc_batch_create": (_int, [C.POINTER(_vp), _int, C.POINTER(_vp)]),
    "fc_batch_destroy": (_int, [_vp]),
    "fc_batch_project": (_int, [_vp, _dp, _int, _dbl, _dbl, C.POINTER(FcResult)]),
    "fc_batch_get_stream": (_int, [_vp, C.POINTER(_vp)]),
}

_lib = None


class FluidCudaError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class FluidInvalidArgument(FluidCudaError, ValueError):
    """The reference throws std::invalid_argument for these."""


class FluidLifecycleError(FluidCudaError):
    """The reference throws std::logic_error for these."""


def lib():
    """Loads libfluidcuda.so, failing loudly when it is absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBRARY):
            raise ImportError(f"libfluidcuda.so is not built ({LIBRARY}); run fluidsim_b200/build.py")
        L = C.CDLL(LIBRARY)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int):
    if status == FC_OK:
        return
    message = lib().fc_last_error().decode(errors="replace")
    if status == 1:
        raise FluidInvalidArgument(status, message)
    if status == 2:
        raise FluidLifecycleError(status, message)
    raise FluidCudaError(status, message)


def kernel_launches() -> int:
    return int(lib().fc_kernel_launches())


def set_launch_mode(mode: str):
    """'graph' (default: one CUDA graph per projection) or 'stream' (host-driven launches)."""
    check(lib().fc_set_launch_mode({"graph": 0, "stream": 1}[mode]))
