"""Python mirror of HighMap's ``hmap::gpu`` erosion interface.

Same names, argument meaning, defaults and in-place behaviour as the C++
functions they stand for (HighMap/include/highmap/erosion.hpp):

* ``init_opencl()``                         gpu_opencl.hpp:166
* ``thermal(z, talus, iterations, bedrock, deposition_map, mask=None)``
                                            erosion.hpp:1784-1801
* ``hydraulic_vpipes(z, water_height, ...)`` erosion.hpp:1206-1223

A grid is a C-contiguous float32 numpy array of shape (ny, nx), so element
(i, j) of the reference's ``hmap::Array`` is ``a[j, i]``.  ``z`` is updated
in place (the reference takes ``Array &z``); optional outputs are arrays the
caller passes to be overwritten (the reference's ``Array *p_...``).

Every call goes through libhm_erosion.so on the GPU.  Device-resident
variants (``thermal_device``, ``hydraulic_vpipes_device``) take torch CUDA
tensors and run on the current torch stream without synchronising.
"""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np

from . import _lib as L
from ._lib import HMError, ThermalOptions, VpipesParams  # noqa: F401

BEDROCK_INTENDED = L.HM_BEDROCK_INTENDED
BEDROCK_LITERAL = L.HM_BEDROCK_LITERAL

_tls = threading.local()


class Context:
    """A CUDA stream plus a device workspace on one GPU (hm_context)."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        L.check(L.lib().hm_context_create(C.byref(self._h), int(device)))
        self.device = int(device)

    @property
    def handle(self):
        return self._h

    def trim(self):
        L.check(L.lib().hm_context_trim(self._h))

    def close(self):
        if self._h:
            L.lib().hm_context_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def default_context() -> Context:
    ctx = getattr(_tls, "ctx", None)
    if ctx is None:
        ctx = Context(0)
        _tls.ctx = ctx
    return ctx


def init_opencl() -> bool:
    """True when a B200-class device is ready (replaces the OpenCL init)."""
    return L.lib().hm_init() == L.HM_OK


def _grid(a, name, shape=None, writable=False):
    if not isinstance(a, np.ndarray) or a.dtype != np.float32 or a.ndim != 2:
        raise TypeError("%s must be a 2-D float32 numpy array" % name)
    if not a.flags.c_contiguous:
        raise ValueError("%s must be C-contiguous" % name)
    if writable and not a.flags.writeable:
        raise ValueError("%s must be writable" % name)
    if shape is not None and a.shape != shape:
        raise ValueError("%s has shape %s, expected %s" % (name, a.shape, shape))
    return a


def _ptr(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def thermal_options(bedrock_mode: int = BEDROCK_INTENDED, time_block: int = 0) -> ThermalOptions:
    o = ThermalOptions()
    L.lib().hm_thermal_default_options(C.byref(o))
    o.bedrock_mode = int(bedrock_mode)
    o.time_block = int(time_block)
    return o


def thermal(z: np.ndarray, talus, iterations: int = 10, bedrock: np.ndarray | None = None,
            deposition_map: np.ndarray | None = None, mask: np.ndarray | None = None,
            bedrock_mode: int = BEDROCK_INTENDED, time_block: int = 0,
            ctx: Context | None = None) -> None:
    """Thermal erosion in place.  ``talus`` is a grid or a float (the
    reference's two overloads); ``mask`` selects the masked overload."""
    _grid(z, "z", writable=True)
    shape = z.shape
    ny, nx = shape
    ctx = ctx or default_context()
    opts = thermal_options(bedrock_mode, time_block)
    if bedrock is not None:
        _grid(bedrock, "bedrock", shape)
    if deposition_map is not None:
        _grid(deposition_map, "deposition_map", shape, writable=True)
    lib = L.lib()
    if np.isscalar(talus) or (isinstance(talus, np.ndarray) and talus.ndim == 0):
        if mask is not None:
            talus = np.full(shape, float(talus), dtype=np.float32)
        else:
            L.check(lib.hm_thermal_scalar(ctx.handle, _ptr(z), nx, ny, C.c_float(float(talus)), int(iterations),
                                          _ptr(bedrock), _ptr(deposition_map), C.byref(opts)))
            return
    _grid(talus, "talus", shape)
    if mask is not None:
        _grid(mask, "mask", shape)
        L.check(lib.hm_thermal_masked(ctx.handle, _ptr(z), nx, ny, _ptr(mask), _ptr(talus), int(iterations),
                                      _ptr(bedrock), _ptr(deposition_map), C.byref(opts)))
    else:
        L.check(lib.hm_thermal(ctx.handle, _ptr(z), nx, ny, _ptr(talus), int(iterations), _ptr(bedrock),
                               _ptr(deposition_map), C.byref(opts)))


def thermal_auto_bedrock(z: np.ndarray, talus, iterations: int = 10, deposition_map: np.ndarray | None = None,
                         mask: np.ndarray | None = None, time_block: int = 0,
                         ctx: Context | None = None) -> None:
    """Thermal erosion with the reference's self-built bedrock, in place
    (hmap::gpu::thermal_auto_bedrock, thermal_gpu.cpp:98-152).  ``talus``
    is a grid or a float; ``mask`` selects the masked overload."""
    _grid(z, "z", writable=True)
    shape = z.shape
    ny, nx = shape
    ctx = ctx or default_context()
    opts = thermal_options(BEDROCK_INTENDED, time_block)
    if deposition_map is not None:
        _grid(deposition_map, "deposition_map", shape, writable=True)
    lib = L.lib()
    if np.isscalar(talus) or (isinstance(talus, np.ndarray) and talus.ndim == 0):
        if mask is not None:
            talus = np.full(shape, float(talus), dtype=np.float32)
        else:
            L.check(lib.hm_thermal_auto_bedrock_scalar(ctx.handle, _ptr(z), nx, ny, C.c_float(float(talus)),
                                                       int(iterations), _ptr(deposition_map), C.byref(opts)))
            return
    _grid(talus, "talus", shape)
    if mask is not None:
        _grid(mask, "mask", shape)
        L.check(lib.hm_thermal_auto_bedrock_masked(ctx.handle, _ptr(z), nx, ny, _ptr(mask), _ptr(talus),
                                                   int(iterations), _ptr(deposition_map), C.byref(opts)))
    else:
        L.check(lib.hm_thermal_auto_bedrock(ctx.handle, _ptr(z), nx, ny, _ptr(talus), int(iterations),
                                            _ptr(deposition_map), C.byref(opts)))


def sediment_deposition(z: np.ndarray, talus: np.ndarray, deposition_map: np.ndarray | None = None,
                        max_deposition: float = 0.01, iterations: int = 5, thermal_subiterations: int = 10,
                        mask: np.ndarray | None = None, ctx: Context | None = None) -> None:
    """hmap::gpu::sediment_deposition (deposition.cpp:19-66), in place."""
    _grid(z, "z", writable=True)
    ny, nx = z.shape
    _grid(talus, "talus", z.shape)
    if deposition_map is not None:
        _grid(deposition_map, "deposition_map", z.shape, writable=True)
    if mask is not None:
        _grid(mask, "mask", z.shape)
    ctx = ctx or default_context()
    L.check(L.lib().hm_sediment_deposition(ctx.handle, _ptr(z), nx, ny, _ptr(talus), C.c_float(max_deposition),
                                           int(iterations), int(thermal_subiterations), _ptr(deposition_map),
                                           _ptr(mask)))


def sediment_deposition_device(z, talus, deposition_map=None, max_deposition: float = 0.01, iterations: int = 5,
                               thermal_subiterations: int = 10, mask=None, ctx: Context | None = None,
                               stream=None) -> None:
    ny, nx = z.shape
    ctx = ctx or default_context()
    L.check(L.lib().hm_sediment_deposition_device(ctx.handle, _tptr(z, "z"), nx, ny, _tptr(talus, "talus", z.shape),
                                                  C.c_float(max_deposition), int(iterations),
                                                  int(thermal_subiterations),
                                                  _tptr(deposition_map, "deposition_map", z.shape),
                                                  _tptr(mask, "mask", z.shape), _stream(stream)))


def sediment_layer(z: np.ndarray, talus_layer: np.ndarray, talus_upper_limit: np.ndarray, iterations: int,
                   apply_post_filter: bool = True, deposition_map: np.ndarray | None = None,
                   ctx: Context | None = None) -> None:
    """hmap::gpu::sediment_layer (deposition.cpp:68-113), in place."""
    _grid(z, "z", writable=True)
    ny, nx = z.shape
    _grid(talus_layer, "talus_layer", z.shape)
    _grid(talus_upper_limit, "talus_upper_limit", z.shape)
    if deposition_map is not None:
        _grid(deposition_map, "deposition_map", z.shape, writable=True)
    ctx = ctx or default_context()
    L.check(L.lib().hm_sediment_layer(ctx.handle, _ptr(z), nx, ny, _ptr(talus_layer), _ptr(talus_upper_limit),
                                      int(iterations), 1 if apply_post_filter else 0, _ptr(deposition_map)))


def sediment_layer_device(z, talus_layer, talus_upper_limit, iterations: int, apply_post_filter: bool = True,
                          deposition_map=None, ctx: Context | None = None, stream=None) -> None:
    ny, nx = z.shape
    ctx = ctx or default_context()
    L.check(L.lib().hm_sediment_layer_device(ctx.handle, _tptr(z, "z"), nx, ny,
                                             _tptr(talus_layer, "talus_layer", z.shape),
                                             _tptr(talus_upper_limit, "talus_upper_limit", z.shape),
                                             int(iterations), 1 if apply_post_filter else 0,
                                             _tptr(deposition_map, "deposition_map", z.shape), _stream(stream)))


def snow_post_filter(z: np.ndarray, s: np.ndarray, snow_depth: float, iterations: int,
                     thermal_talus_ratio: float = 0.2, ctx: Context | None = None) -> None:
    """Post-filter of hmap::gpu::snow_simulation (snow_simulation.cpp:140-152
    and its clamp_min(s, 0)): updates the snow depth s over terrain z in place."""
    _grid(z, "z")
    _grid(s, "s", z.shape, writable=True)
    ny, nx = z.shape
    ctx = ctx or default_context()
    L.check(L.lib().hm_snow_post_filter(ctx.handle, _ptr(z), _ptr(s), nx, ny, C.c_float(snow_depth),
                                        int(iterations), C.c_float(thermal_talus_ratio)))


def snow_post_filter_device(z, s, snow_depth: float, iterations: int, thermal_talus_ratio: float = 0.2,
                            ctx: Context | None = None, stream=None) -> None:
    ny, nx = z.shape
    ctx = ctx or default_context()
    L.check(L.lib().hm_snow_post_filter_device(ctx.handle, _tptr(z, "z"), _tptr(s, "s", z.shape), nx, ny,
                                               C.c_float(snow_depth), int(iterations),
                                               C.c_float(thermal_talus_ratio), _stream(stream)))


RIDGE, SCREE, SCHOTT, OLSEN = 0, 1, 2, 3
FLATTEN, INFLATE, RIB = 4, 5, 6


def _sibling_host(z, talus, deposition_map, mask):
    _grid(z, "z", writable=True)
    shape = z.shape
    ny, nx = shape
    _grid(talus, "talus", shape)
    if deposition_map is not None:
        _grid(deposition_map, "deposition_map", shape, writable=True)
    if mask is not None:
        _grid(mask, "mask", shape)
    return nx, ny


def thermal_ridge(z: np.ndarray, talus: np.ndarray, iterations: int = 10, deposition_map: np.ndarray | None = None,
                  mask: np.ndarray | None = None, ctx: Context | None = None) -> None:
    """hmap::gpu::thermal_ridge (thermal_gpu.cpp:274-311), in place."""
    nx, ny = _sibling_host(z, talus, deposition_map, mask)
    ctx = ctx or default_context()
    L.check(L.lib().hm_thermal_ridge(ctx.handle, _ptr(z), nx, ny, _ptr(talus), int(iterations), _ptr(deposition_map),
                                     _ptr(mask)))


def thermal_scree(z: np.ndarray, talus: np.ndarray, zmax: np.ndarray, iterations: int = 10,
                  deposition_map: np.ndarray | None = None, mask: np.ndarray | None = None,
                  ctx: Context | None = None) -> None:
    """hmap::gpu::thermal_scree (thermal_gpu.cpp:355-396), in place."""
    nx, ny = _sibling_host(z, talus, deposition_map, mask)
    _grid(zmax, "zmax", z.shape)
    ctx = ctx or default_context()
    L.check(L.lib().hm_thermal_scree(ctx.handle, _ptr(z), nx, ny, _ptr(talus), _ptr(zmax), int(iterations),
                                     _ptr(deposition_map), _ptr(mask)))


def thermal_schott(z: np.ndarray, talus: np.ndarray, iterations: int = 10, intensity: float = 0.2,
                   deposition_map: np.ndarray | None = None, mask: np.ndarray | None = None,
                   ctx: Context | None = None) -> None:
    """hmap::gpu::thermal_schott (thermal_gpu.cpp:313-353), in place."""
    nx, ny = _sibling_host(z, talus, deposition_map, mask)
    ctx = ctx or default_context()
    L.check(L.lib().hm_thermal_schott(ctx.handle, _ptr(z), nx, ny, _ptr(talus), int(iterations),
                                      C.c_float(intensity), _ptr(deposition_map), _ptr(mask)))


def thermal_olsen(z: np.ndarray, talus: np.ndarray, iterations: int = 10, mask: np.ndarray | None = None,
                  ctx: Context | None = None) -> None:
    """hmap::gpu::thermal_olsen (thermal_gpu.cpp:221-247), in place."""
    nx, ny = _sibling_host(z, talus, None, mask)
    ctx = ctx or default_context()
    L.check(L.lib().hm_thermal_olsen(ctx.handle, _ptr(z), nx, ny, _ptr(talus), int(iterations), _ptr(mask)))


def thermal_stencil_device(rule: int, z, talus, iterations: int = 10, zmax=None, intensity: float = 0.2,
                           deposition_map=None, mask=None, ctx: Context | None = None, stream=None) -> None:
    ny, nx = z.shape
    ctx = ctx or default_context()
    L.check(L.lib().hm_thermal_stencil_device(ctx.handle, int(rule), _tptr(z, "z"), nx, ny,
                                              _tptr(talus, "talus", z.shape), _tptr(zmax, "zmax", z.shape),
                                              C.c_float(intensity), int(iterations),
                                              _tptr(deposition_map, "deposition_map", z.shape),
                                              _tptr(mask, "mask", z.shape), _stream(stream)))


def flow_simulation_viscous(z: np.ndarray, water_height: float, depth_map: np.ndarray, iterations: int,
                            dt: float = 0.5, dry_out_ratio: float = 0.0, viscosity: float = 1.0, power: float = 2.5,
                            ctx: Context | None = None) -> np.ndarray:
    """hmap::gpu::flow_simulation_viscous (flow_simulation.cpp:112-157): the water depth."""
    _grid(z, "z")
    _grid(depth_map, "depth_map", z.shape)
    ny, nx = z.shape
    out = np.empty_like(z)
    ctx = ctx or default_context()
    L.check(L.lib().hm_flow_simulation_viscous(ctx.handle, _ptr(z), nx, ny, C.c_float(water_height), _ptr(depth_map),
                                               int(iterations), C.c_float(dt), C.c_float(dry_out_ratio),
                                               C.c_float(viscosity), C.c_float(power), _ptr(out)))
    return out


def flow_simulation_viscous_device(z, water_height: float, depth_map, iterations: int, water_depth, dt: float = 0.5,
                                   dry_out_ratio: float = 0.0, viscosity: float = 1.0, power: float = 2.5,
                                   ctx: Context | None = None, stream=None) -> None:
    ny, nx = z.shape
    ctx = ctx or default_context()
    L.check(L.lib().hm_flow_simulation_viscous_device(ctx.handle, _tptr(z, "z"), nx, ny, C.c_float(water_height),
                                                      _tptr(depth_map, "depth_map", z.shape), int(iterations),
                                                      C.c_float(dt), C.c_float(dry_out_ratio), C.c_float(viscosity),
                                                      C.c_float(power), _tptr(water_depth, "water_depth", z.shape),
                                                      _stream(stream)))


def thermal_flatten(z: np.ndarray, talus: np.ndarray, iterations: int, sigma_inf: float = 0.5,
                    sigma_sup: float = 0.0, mask: np.ndarray | None = None, ctx: Context | None = None) -> None:
    """hmap::gpu::thermal_flatten (thermal_gpu.cpp:154-190), in place."""
    nx, ny = _sibling_host(z, talus, None, mask)
    ctx = ctx or default_context()
    L.check(L.lib().hm_thermal_flatten(ctx.handle, _ptr(z), nx, ny, _ptr(talus), int(iterations),
                                       C.c_float(sigma_inf), C.c_float(sigma_sup), _ptr(mask)))


def thermal_inflate(z: np.ndarray, talus: np.ndarray, iterations: int = 10, mask: np.ndarray | None = None,
                    ctx: Context | None = None) -> None:
    """hmap::gpu::thermal_inflate (thermal_gpu.cpp:192-219), in place."""
    nx, ny = _sibling_host(z, talus, None, mask)
    ctx = ctx or default_context()
    L.check(L.lib().hm_thermal_inflate(ctx.handle, _ptr(z), nx, ny, _ptr(talus), int(iterations), _ptr(mask)))


def thermal_rib(z: np.ndarray, iterations: int, mask: np.ndarray | None = None, ctx: Context | None = None) -> None:
    """hmap::gpu::thermal_rib (thermal_gpu.cpp:249-272), in place."""
    _grid(z, "z", writable=True)
    ny, nx = z.shape
    if mask is not None:
        _grid(mask, "mask", z.shape)
    ctx = ctx or default_context()
    L.check(L.lib().hm_thermal_rib(ctx.handle, _ptr(z), nx, ny, int(iterations), _ptr(mask)))


def thermal_relief_device(rule: int, z, talus=None, iterations: int = 10, sigma_inf: float = 0.5,
                          sigma_sup: float = 0.0, mask=None, ctx: Context | None = None, stream=None) -> None:
    ny, nx = z.shape
    ctx = ctx or default_context()
    L.check(L.lib().hm_thermal_relief_device(ctx.handle, int(rule), _tptr(z, "z"), nx, ny,
                                             _tptr(talus, "talus", z.shape), C.c_float(sigma_inf),
                                             C.c_float(sigma_sup), int(iterations), _tptr(mask, "mask", z.shape),
                                             _stream(stream)))


def flow_simulation(z: np.ndarray, water_height: float, depth_map: np.ndarray, iterations: int, dt: float = 0.5,
                    flux_diffusion: bool = True, flux_diffusion_strength: float = 0.01, dry_out_ratio: float = 0.0,
                    ctx: Context | None = None) -> np.ndarray:
    """Water depth of the pipe model's flow and water passes on the fixed
    terrain z (hmap::gpu::flow_simulation, flow_simulation.cpp:26-110)."""
    _grid(z, "z")
    shape = z.shape
    ny, nx = shape
    _grid(depth_map, "depth_map", shape)
    out = np.empty_like(z)
    ctx = ctx or default_context()
    L.check(L.lib().hm_flow_simulation(ctx.handle, _ptr(z), nx, ny, C.c_float(water_height), _ptr(depth_map),
                                       int(iterations), C.c_float(dt), int(bool(flux_diffusion)),
                                       C.c_float(flux_diffusion_strength), C.c_float(dry_out_ratio), _ptr(out)))
    return out


def vpipes_params(**kw) -> VpipesParams:
    p = VpipesParams()
    L.lib().hm_vpipes_default_params(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise TypeError("unknown vpipes parameter %r" % k)
        setattr(p, k, int(v) if isinstance(v, bool) else v)
    return p


def hydraulic_vpipes(z: np.ndarray, water_height: float = 1e-2, maintain_water_volume: bool = True,
                     evap_rate: float = 0.1, iterations: int = 50, dt: float = 0.5,
                     k_capacity: float = 0.5, k_erode: float = 0.001, k_depose: float = 0.01,
                     k_discharge_exp: float = 1.0, downcutting_max_depth_ratio: float = 10.0,
                     flux_diffusion: bool = True, flux_diffusion_strength: float = 0.01,
                     rain_map: np.ndarray | None = None, water_depth: np.ndarray | None = None,
                     sediment: np.ndarray | None = None, vel_u: np.ndarray | None = None,
                     vel_v: np.ndarray | None = None, *, gravity: float = 1.0, pipe_length: float = 1.0,
                     pipe_area: float = 1.0, rain_per_step: float = 0.0, initial_water: float = -1.0,
                     ctx: Context | None = None) -> None:
    """Virtual-pipes hydraulic erosion in place (reference defaults); the
    keyword-only extensions default to the reference's behaviour."""
    _grid(z, "z", writable=True)
    shape = z.shape
    ny, nx = shape
    for name, a in (("rain_map", rain_map),):
        if a is not None:
            _grid(a, name, shape)
    for name, a in (("water_depth", water_depth), ("sediment", sediment), ("vel_u", vel_u), ("vel_v", vel_v)):
        if a is not None:
            _grid(a, name, shape, writable=True)
    p = vpipes_params(water_height=water_height, maintain_water_volume=maintain_water_volume,
                      evap_rate=evap_rate, iterations=iterations, dt=dt, k_capacity=k_capacity,
                      k_erode=k_erode, k_depose=k_depose, k_discharge_exp=k_discharge_exp,
                      downcutting_max_depth_ratio=downcutting_max_depth_ratio,
                      flux_diffusion=flux_diffusion, flux_diffusion_strength=flux_diffusion_strength,
                      gravity=gravity, pipe_length=pipe_length, pipe_area=pipe_area,
                      rain_per_step=rain_per_step, initial_water=initial_water)
    ctx = ctx or default_context()
    L.check(L.lib().hm_vpipes(ctx.handle, _ptr(z), nx, ny, C.byref(p), _ptr(rain_map), _ptr(water_depth),
                              _ptr(sediment), _ptr(vel_u), _ptr(vel_v)))


# ---- device-resident (torch CUDA tensors) --------------------------------

def _tptr(t, name, shape=None):
    if t is None:
        return None
    import torch
    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float32:
        raise TypeError("%s must be a float32 CUDA tensor" % name)
    if not t.is_contiguous():
        raise ValueError("%s must be contiguous" % name)
    if shape is not None and tuple(t.shape) != tuple(shape):
        raise ValueError("%s has shape %s, expected %s" % (name, tuple(t.shape), tuple(shape)))
    return C.c_void_p(t.data_ptr())


def _stream(stream):
    if stream is not None:
        return C.c_void_p(int(stream))
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def thermal_device(z, talus, iterations: int = 10, bedrock=None, deposition_map=None, mask=None,
                   bedrock_mode: int = BEDROCK_INTENDED, time_block: int = 0, ctx: Context | None = None,
                   stream=None) -> None:
    ny, nx = z.shape
    zp = _tptr(z, "z")
    ctx = ctx or default_context()
    opts = thermal_options(bedrock_mode, time_block)
    if isinstance(talus, (int, float)):
        tp, tv = None, float(talus)
    else:
        tp, tv = _tptr(talus, "talus", z.shape), 0.0
    L.check(L.lib().hm_thermal_device(ctx.handle, zp, nx, ny, tp, C.c_float(tv), int(iterations),
                                      _tptr(bedrock, "bedrock", z.shape),
                                      _tptr(deposition_map, "deposition_map", z.shape),
                                      _tptr(mask, "mask", z.shape), C.byref(opts), _stream(stream)))


def thermal_auto_bedrock_device(z, talus, iterations: int = 10, deposition_map=None, mask=None,
                                time_block: int = 0, ctx: Context | None = None, stream=None) -> None:
    ny, nx = z.shape
    zp = _tptr(z, "z")
    ctx = ctx or default_context()
    opts = thermal_options(BEDROCK_INTENDED, time_block)
    if isinstance(talus, (int, float)):
        tp, tv = None, float(talus)
    else:
        tp, tv = _tptr(talus, "talus", z.shape), 0.0
    L.check(L.lib().hm_thermal_auto_bedrock_device(ctx.handle, zp, nx, ny, tp, C.c_float(tv), int(iterations),
                                                   _tptr(deposition_map, "deposition_map", z.shape),
                                                   _tptr(mask, "mask", z.shape), C.byref(opts),
                                                   _stream(stream)))


def flow_simulation_device(z, water_height: float, depth_map, iterations: int, out, dt: float = 0.5,
                           flux_diffusion: bool = True, flux_diffusion_strength: float = 0.01,
                           dry_out_ratio: float = 0.0, ctx: Context | None = None, stream=None) -> None:
    ny, nx = z.shape
    ctx = ctx or default_context()
    L.check(L.lib().hm_flow_simulation_device(ctx.handle, _tptr(z, "z"), nx, ny, C.c_float(water_height),
                                              _tptr(depth_map, "depth_map", z.shape), int(iterations),
                                              C.c_float(dt), int(bool(flux_diffusion)),
                                              C.c_float(flux_diffusion_strength), C.c_float(dry_out_ratio),
                                              _tptr(out, "out", z.shape), _stream(stream)))


def hydraulic_vpipes_device(z, params: VpipesParams | None = None, rain_map=None, water_depth=None,
                            sediment=None, vel_u=None, vel_v=None, ctx: Context | None = None,
                            stream=None) -> None:
    ny, nx = z.shape
    ctx = ctx or default_context()
    p = params if params is not None else vpipes_params()
    L.check(L.lib().hm_vpipes_device(ctx.handle, _tptr(z, "z"), nx, ny, C.byref(p),
                                     _tptr(rain_map, "rain_map", z.shape),
                                     _tptr(water_depth, "water_depth", z.shape),
                                     _tptr(sediment, "sediment", z.shape), _tptr(vel_u, "vel_u", z.shape),
                                     _tptr(vel_v, "vel_v", z.shape), _stream(stream)))


def vpipes_set_launch(tpb: int = 0, radius: int = 2, rows: int = 128) -> None:
    """Launch shape of the fused vpipes step (tpb=0: built-in choice)."""
    L.check(L.lib().hm_vpipes_set_launch(int(tpb), int(radius), int(rows)))


VPIPES_AUTO, VPIPES_TILED, VPIPES_STREAMING, VPIPES_TILED_CP_ASYNC, VPIPES_TILED_TB2 = -1, 0, 1, 2, 3


def vpipes_set_algorithm(algo: int = VPIPES_AUTO) -> None:
    """Step kernels of the vpipes solver (tiled with TMA staging where the
    grid allows it, tiled with cp.async staging, streaming, or auto)."""
    L.check(L.lib().hm_vpipes_set_algorithm(int(algo)))


def debug_tma_expect_extra(nbytes: int = 0) -> None:
    """Test hook: every TMA-staged vpipes tile expects ``nbytes`` more than
    its boxes deliver, so its bounded wait runs out and the call reports
    HM_ERR_TIMEOUT (0 turns it off)."""
    L.check(L.lib().hm_debug_tma_expect_extra(int(nbytes)))


def thermal_set_launch(rows: int = 0) -> None:
    """Output rows per CTA of the blocked thermal kernel (0: built-in)."""
    L.check(L.lib().hm_thermal_set_launch(int(rows)))


def launch_count() -> int:
    return int(L.lib().hm_launch_count())


def launch_count_reset() -> None:
    L.lib().hm_launch_count_reset()
