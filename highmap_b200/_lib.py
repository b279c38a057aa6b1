"""Loader of libhm_erosion.so and its ctypes signatures.

The library is the only compute path: if it is missing or cannot load,
every call raises; nothing falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libhm_erosion.so")

HM_OK = 0
HM_ERR_INVALID_ARGUMENT = 1
HM_ERR_NO_DEVICE = 2
HM_ERR_OUT_OF_MEMORY = 3
HM_ERR_CUDA = 4
HM_ERR_TIMEOUT = 5
HM_ERR_BUSY = 6

HM_BEDROCK_INTENDED = 0
HM_BEDROCK_LITERAL = 1

# every symbol include/hm_erosion.h declares (checked by the CPU tests)
EXPORTED = (
    "hm_init", "hm_context_create", "hm_context_destroy", "hm_context_trim",
    "hm_status_string", "hm_last_error", "hm_thermal_default_options",
    "hm_thermal", "hm_thermal_scalar", "hm_thermal_masked", "hm_thermal_device",
    "hm_thermal_auto_bedrock", "hm_thermal_auto_bedrock_scalar", "hm_thermal_auto_bedrock_masked",
    "hm_thermal_auto_bedrock_device", "hm_flow_simulation", "hm_flow_simulation_device",
    "hm_thermal_ridge", "hm_thermal_scree", "hm_thermal_schott", "hm_thermal_olsen", "hm_thermal_stencil_device",
    "hm_sediment_deposition", "hm_sediment_deposition_device", "hm_sediment_layer", "hm_sediment_layer_device",
    "hm_snow_post_filter", "hm_snow_post_filter_device",
    "hm_thermal_flatten", "hm_thermal_inflate", "hm_thermal_rib", "hm_thermal_relief_device",
    "hm_flow_simulation_viscous", "hm_flow_simulation_viscous_device",
    "hm_vpipes_default_params", "hm_vpipes", "hm_vpipes_device",
    "hm_launch_count", "hm_launch_count_reset",
    "hm_thermal_device_noalloc", "hm_vpipes_set_launch", "hm_thermal_set_launch",
    "hm_batch_create", "hm_batch_destroy", "hm_batch_job_bytes", "hm_batch_add", "hm_batch_step",
    "hm_batch_synchronize", "hm_batch_job_status", "hm_batch_release", "hm_batch_bytes_in_use",
    "hm_batch_round", "hm_batch_run",
    "hm_autotune", "hm_autotune_save", "hm_autotune_load", "hm_autotune_clear", "hm_vpipes_set_algorithm",
    "hm_debug_tma_expect_extra", "hm_batch_snapshot_bytes", "hm_batch_evict", "hm_batch_restore",
)

HM_JOB_THERMAL = 1
HM_JOB_VPIPES = 2


class HMError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__("%s (status %d)" % (message, status))
        self.status = status


class ThermalOptions(C.Structure):
    _fields_ = [("bedrock_mode", C.c_int), ("time_block", C.c_int)]


class VpipesParams(C.Structure):
    """hm_vpipes_params: the reference's hydraulic_vpipes parameters
    (HighMap/include/highmap/erosion.hpp:1206-1223) and the extensions."""

    _fields_ = [
        ("water_height", C.c_float),
        ("maintain_water_volume", C.c_int),
        ("evap_rate", C.c_float),
        ("iterations", C.c_int),
        ("dt", C.c_float),
        ("k_capacity", C.c_float),
        ("k_erode", C.c_float),
        ("k_depose", C.c_float),
        ("k_discharge_exp", C.c_float),
        ("downcutting_max_depth_ratio", C.c_float),
        ("flux_diffusion", C.c_int),
        ("flux_diffusion_strength", C.c_float),
        ("gravity", C.c_float),
        ("pipe_length", C.c_float),
        ("pipe_area", C.c_float),
        ("rain_per_step", C.c_float),
        ("initial_water", C.c_float),
    ]


class TuneResult(C.Structure):
    _fields_ = [("tpb", C.c_int), ("radius", C.c_int), ("rows", C.c_int), ("time_block", C.c_int),
                ("ms_per_step", C.c_float), ("candidates", C.c_int)]


class Job(C.Structure):
    """hm_job: one solve of a batch (device pointers)."""

    _fields_ = [
        ("kind", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("iterations", C.c_int),
        ("z", C.c_void_p),
        ("talus", C.c_void_p), ("talus_value", C.c_float), ("bedrock", C.c_void_p), ("bedrock_mode", C.c_int),
        ("deposition_map", C.c_void_p),
        ("vpipes", VpipesParams),
        ("rain_map", C.c_void_p), ("water_depth", C.c_void_p), ("sediment", C.c_void_p),
        ("vel_u", C.c_void_p), ("vel_v", C.c_void_p),
    ]


_lock = threading.Lock()
_lib = None


def _declare(lib):
    vp = C.c_void_p
    i = C.c_int
    f = C.c_float
    lib.hm_init.restype = i
    lib.hm_context_create.argtypes = [C.POINTER(vp), i]
    lib.hm_context_destroy.argtypes = [vp]
    lib.hm_context_trim.argtypes = [vp]
    lib.hm_status_string.restype = C.c_char_p
    lib.hm_status_string.argtypes = [i]
    lib.hm_last_error.restype = C.c_char_p
    lib.hm_thermal_default_options.argtypes = [vp]
    lib.hm_thermal.argtypes = [vp, vp, i, i, vp, i, vp, vp, vp]
    lib.hm_thermal_scalar.argtypes = [vp, vp, i, i, f, i, vp, vp, vp]
    lib.hm_thermal_masked.argtypes = [vp, vp, i, i, vp, vp, i, vp, vp, vp]
    lib.hm_thermal_device.argtypes = [vp, vp, i, i, vp, f, i, vp, vp, vp, vp, vp]
    lib.hm_thermal_auto_bedrock.argtypes = [vp, vp, i, i, vp, i, vp, vp]
    lib.hm_thermal_auto_bedrock_scalar.argtypes = [vp, vp, i, i, f, i, vp, vp]
    lib.hm_thermal_auto_bedrock_masked.argtypes = [vp, vp, i, i, vp, vp, i, vp, vp]
    lib.hm_thermal_auto_bedrock_device.argtypes = [vp, vp, i, i, vp, f, i, vp, vp, vp, vp]
    lib.hm_flow_simulation.argtypes = [vp, vp, i, i, f, vp, i, f, i, f, f, vp]
    lib.hm_thermal_ridge.argtypes = [vp, vp, i, i, vp, i, vp, vp]
    lib.hm_sediment_deposition.argtypes = [vp, vp, i, i, vp, f, i, i, vp, vp]
    lib.hm_sediment_deposition_device.argtypes = [vp, vp, i, i, vp, f, i, i, vp, vp, vp]
    lib.hm_sediment_layer.argtypes = [vp, vp, i, i, vp, vp, i, i, vp]
    lib.hm_sediment_layer_device.argtypes = [vp, vp, i, i, vp, vp, i, i, vp, vp]
    lib.hm_snow_post_filter.argtypes = [vp, vp, vp, i, i, f, i, f]
    lib.hm_snow_post_filter_device.argtypes = [vp, vp, vp, i, i, f, i, f, vp]
    lib.hm_thermal_flatten.argtypes = [vp, vp, i, i, vp, i, f, f, vp]
    lib.hm_thermal_inflate.argtypes = [vp, vp, i, i, vp, i, vp]
    lib.hm_thermal_rib.argtypes = [vp, vp, i, i, i, vp]
    lib.hm_thermal_relief_device.argtypes = [vp, i, vp, i, i, vp, f, f, i, vp, vp]
    lib.hm_flow_simulation_viscous.argtypes = [vp, vp, i, i, f, vp, i, f, f, f, f, vp]
    lib.hm_flow_simulation_viscous_device.argtypes = [vp, vp, i, i, f, vp, i, f, f, f, f, vp, vp]
    lib.hm_thermal_scree.argtypes = [vp, vp, i, i, vp, vp, i, vp, vp]
    lib.hm_thermal_schott.argtypes = [vp, vp, i, i, vp, i, f, vp, vp]
    lib.hm_thermal_olsen.argtypes = [vp, vp, i, i, vp, i, vp]
    lib.hm_thermal_stencil_device.argtypes = [vp, i, vp, i, i, vp, vp, f, i, vp, vp, vp]
    lib.hm_flow_simulation_device.argtypes = [vp, vp, i, i, f, vp, i, f, i, f, f, vp, vp]
    lib.hm_vpipes_default_params.argtypes = [vp]
    lib.hm_vpipes.argtypes = [vp, vp, i, i, vp, vp, vp, vp, vp, vp]
    lib.hm_vpipes_device.argtypes = [vp, vp, i, i, vp, vp, vp, vp, vp, vp, vp]
    lib.hm_launch_count.restype = C.c_ulonglong
    lib.hm_thermal_device_noalloc.argtypes = [vp, i, i, vp, f, i, vp, i, vp]
    lib.hm_vpipes_set_launch.argtypes = [i, i, i]
    lib.hm_thermal_set_launch.argtypes = [i]
    lib.hm_batch_create.argtypes = [vp, C.POINTER(vp)]
    lib.hm_batch_destroy.argtypes = [vp]
    lib.hm_batch_job_bytes.argtypes = [vp]
    lib.hm_batch_job_bytes.restype = C.c_size_t
    lib.hm_batch_add.argtypes = [vp, vp, C.POINTER(i)]
    lib.hm_batch_step.argtypes = [vp, i]
    lib.hm_batch_synchronize.argtypes = [vp]
    lib.hm_batch_job_status.argtypes = [vp, i, C.POINTER(i), C.POINTER(i)]
    lib.hm_batch_release.argtypes = [vp, i]
    lib.hm_batch_bytes_in_use.argtypes = [vp]
    lib.hm_batch_bytes_in_use.restype = C.c_size_t
    lib.hm_batch_snapshot_bytes.argtypes = [vp, i]
    lib.hm_batch_snapshot_bytes.restype = C.c_size_t
    lib.hm_batch_evict.argtypes = [vp, i, vp]
    lib.hm_batch_restore.argtypes = [vp, i, vp]
    lib.hm_batch_round.argtypes = [vp]
    lib.hm_batch_round.restype = C.c_longlong
    lib.hm_batch_run.argtypes = [vp, vp, i, i]
    lib.hm_autotune.argtypes = [vp, i, i, i, i, vp]
    lib.hm_vpipes_set_algorithm.argtypes = [i]
    lib.hm_debug_tma_expect_extra.argtypes = [C.c_uint]
    lib.hm_autotune_save.argtypes = [C.c_char_p]
    lib.hm_autotune_load.argtypes = [C.c_char_p, C.POINTER(i)]
    for name in EXPORTED:
        getattr(lib, name)  # raises AttributeError if a symbol is missing
    return lib


def lib():
    """The loaded library; raises if it is not built."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise RuntimeError(
                        "libhm_erosion.so is not built (expected at %s); run "
                        "`python -m highmap_b200.build`" % LIB_PATH)
                _lib = _declare(C.CDLL(LIB_PATH))
    return _lib


def check(status: int) -> None:
    if status != HM_OK:
        msg = lib().hm_last_error().decode(errors="replace") or lib().hm_status_string(status).decode()
        raise HMError(status, msg)
