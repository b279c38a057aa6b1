"""ctypes front-end of the CPU oracle and of the reference checker.

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
CPU-baseline legs of bench.py, always as the checker or the timed CPU
baseline, never as the product path.  Grids are 2-D numpy arrays of shape
(ny, nx), C order, so element (i, j) of the reference's hmap::Array is
``a[j, i]``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build_oracle as _b

BEDROCK_INTENDED = 0
BEDROCK_LITERAL = 1


class VpipesParams(C.Structure):
    """Mirror of hmo_vpipes_params (hm_oracle.h) and of the product's
    hm_vpipes_params: the reference parameters of erosion.hpp:1206-1223 plus
    the extensions gravity, pipe_length, pipe_area, rain_per_step and
    initial_water (defaults reproduce the reference)."""

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

    @classmethod
    def make(cls, **kw):
        p = cls()
        _lib().hmo_vpipes_default_params(C.byref(p))
        for k, v in kw.items():
            if not hasattr(p, k):
                raise KeyError(k)
            setattr(p, k, v)
        return p

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_LIB = None
_REF = None


def _lib():
    global _LIB
    if _LIB is None:
        _LIB = C.CDLL(_b.build_oracle())
        _LIB.hmo_vpipes_default_params.argtypes = [C.c_void_p]
        _LIB.hmo_sample_linear_mirror_f32.restype = C.c_float
        _LIB.hmo_sample_linear_mirror_f32.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float]
    return _LIB


def ref_available() -> bool:
    return os.path.exists(_b.REF_SO) or _b.build_ref() is not None


def _ref():
    global _REF
    if _REF is None:
        path = _b.build_ref()
        if path is None:
            raise RuntimeError("reference checker oracle/_ref/libhm_ref.so is not built")
        _REF = C.CDLL(path)
    return _REF


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _grid(a, dtype):
    a = np.ascontiguousarray(a, dtype=dtype)
    if a.ndim != 2:
        raise ValueError("expected a 2-D grid")
    return a


def _out(like, want):
    return np.empty_like(like) if want else None


def thermal(z, talus, iterations, bedrock=None, mask=None, deposition=False,
            bedrock_mode=BEDROCK_INTENDED, dtype=np.float32):
    """Oracle thermal; returns (z, deposition_map or None)."""
    z = _grid(z, dtype).copy()
    ny, nx = z.shape
    if np.isscalar(talus):
        talus = np.full_like(z, talus)
    talus = _grid(talus, dtype)
    bedrock = None if bedrock is None else _grid(bedrock, dtype)
    mask = None if mask is None else _grid(mask, dtype)
    depo = _out(z, deposition)
    fn = _lib().hmo_thermal_f32 if dtype == np.float32 else _lib().hmo_thermal_f64
    rc = fn(_p(z), nx, ny, _p(talus), int(iterations), _p(bedrock), _p(depo), _p(mask), int(bedrock_mode))
    if rc:
        raise ValueError("oracle thermal rejected its arguments (status %d)" % rc)
    return z, depo


def thermal_auto_bedrock(z, talus, iterations, deposition=False):
    z = _grid(z, np.float32).copy()
    ny, nx = z.shape
    if np.isscalar(talus):
        talus = np.full_like(z, talus)
    talus = _grid(talus, np.float32)
    depo = _out(z, deposition)
    rc = _lib().hmo_thermal_auto_bedrock_f32(_p(z), nx, ny, _p(talus), int(iterations), _p(depo))
    if rc:
        raise ValueError("oracle thermal_auto_bedrock rejected its arguments (status %d)" % rc)
    return z, depo


def vpipes(z, params: VpipesParams, rain_map=None, dtype=np.float32):
    """Oracle vpipes; returns (z, water_depth, sediment, vel_u, vel_v)."""
    z = _grid(z, dtype).copy()
    ny, nx = z.shape
    rain = None if rain_map is None else _grid(rain_map, dtype)
    outs = [np.empty_like(z) for _ in range(4)]
    fn = _lib().hmo_vpipes_f32 if dtype == np.float32 else _lib().hmo_vpipes_f64
    rc = fn(_p(z), nx, ny, C.byref(params), _p(rain), *[_p(o) for o in outs])
    if rc:
        raise ValueError("oracle vpipes rejected its arguments (status %d)" % rc)
    return (z, *outs)


def sediment_deposition(z, talus, max_deposition=0.01, iterations=5, thermal_subiterations=10, mask=None,
                        dtype=np.float32):
    """Oracle sediment_deposition; returns (z, deposition map)."""
    z = _grid(z, dtype).copy()
    ny, nx = z.shape
    talus = _grid(talus, dtype)
    mask = None if mask is None else _grid(mask, dtype)
    depo = np.empty_like(z)
    fn = _lib().hmo_sediment_deposition_f32 if dtype == np.float32 else _lib().hmo_sediment_deposition_f64
    S = C.c_float if dtype == np.float32 else C.c_double
    rc = fn(_p(z), nx, ny, _p(talus), S(max_deposition), int(iterations), int(thermal_subiterations), _p(depo),
            _p(mask))
    if rc:
        raise ValueError("oracle sediment_deposition rejected its arguments (status %d)" % rc)
    return z, depo


def ref_sediment_deposition(z, talus, max_deposition=0.01, iterations=5, thermal_subiterations=10, mask=None):
    """deposition.cpp:19-66 driven over the reference's thermal kernel text."""
    z = _grid(z, np.float32).copy()
    ny, nx = z.shape
    talus = _grid(talus, np.float32)
    mask = None if mask is None else _grid(mask, np.float32)
    depo = np.empty_like(z)
    rc = _ref().ref_sediment_deposition(_p(z), nx, ny, _p(talus), C.c_float(max_deposition), int(iterations),
                                        int(thermal_subiterations), _p(depo), _p(mask))
    if rc:
        raise ValueError("ref sediment_deposition rejected its arguments (status %d)" % rc)
    return z, depo


def sediment_layer(z, talus_layer, talus_upper_limit, iterations, apply_post_filter=True, dtype=np.float32):
    """Oracle sediment_layer (deposition.cpp:68-113); returns (z, deposition map)."""
    z = _grid(z, dtype).copy()
    ny, nx = z.shape
    tl = _grid(talus_layer, dtype)
    tu = _grid(talus_upper_limit, dtype)
    depo = np.empty_like(z)
    fn = _lib().hmo_sediment_layer_f32 if dtype == np.float32 else _lib().hmo_sediment_layer_f64
    rc = fn(_p(z), nx, ny, _p(tl), _p(tu), int(iterations), 1 if apply_post_filter else 0, _p(depo))
    if rc:
        raise ValueError("oracle sediment_layer rejected its arguments (status %d)" % rc)
    return z, depo


def ref_sediment_layer(z, talus_layer, talus_upper_limit, iterations, apply_post_filter=True):
    """deposition.cpp:68-113 driven over the reference's thermal kernel text."""
    z = _grid(z, np.float32).copy()
    ny, nx = z.shape
    tl = _grid(talus_layer, np.float32)
    tu = _grid(talus_upper_limit, np.float32)
    depo = np.empty_like(z)
    rc = _ref().ref_sediment_layer(_p(z), nx, ny, _p(tl), _p(tu), int(iterations), 1 if apply_post_filter else 0,
                                   _p(depo))
    if rc:
        raise ValueError("ref sediment_layer rejected its arguments (status %d)" % rc)
    return z, depo


def snow_post_filter(z, s, snow_depth, iterations, thermal_talus_ratio, dtype=np.float32):
    """Oracle snow_simulation post-filter (snow_simulation.cpp:140-152 and
    its clamp_min(s, 0)); returns the new snow depth."""
    z = _grid(z, dtype)
    s = _grid(s, dtype).copy()
    ny, nx = z.shape
    fn = _lib().hmo_snow_post_filter_f32 if dtype == np.float32 else _lib().hmo_snow_post_filter_f64
    S = C.c_float if dtype == np.float32 else C.c_double
    rc = fn(_p(z), _p(s), nx, ny, S(snow_depth), int(iterations), S(thermal_talus_ratio))
    if rc:
        raise ValueError("oracle snow_post_filter rejected its arguments (status %d)" % rc)
    return s


def ref_snow_post_filter(z, s, snow_depth, iterations, thermal_talus_ratio):
    """snow_simulation.cpp:140-152 driven over the reference's thermal kernel text."""
    z = _grid(z, np.float32)
    s = _grid(s, np.float32).copy()
    ny, nx = z.shape
    rc = _ref().ref_snow_post_filter(_p(z), _p(s), nx, ny, C.c_float(snow_depth), int(iterations),
                                     C.c_float(thermal_talus_ratio))
    if rc:
        raise ValueError("ref snow_post_filter rejected its arguments (status %d)" % rc)
    return s


FLATTEN, INFLATE, RIB = 4, 5, 6


def thermal_relief(rule, z, talus=None, iterations=10, sigma_inf=0.5, sigma_sup=0.0, mask=None, dtype=np.float32):
    """Oracle thermal_flatten (rule 4) / thermal_inflate (5) / thermal_rib (6)
    (thermal_gpu.cpp:154-219,249-272); returns z."""
    z = _grid(z, dtype).copy()
    ny, nx = z.shape
    talus = None if talus is None else _grid(talus, dtype)
    mask = None if mask is None else _grid(mask, dtype)
    fn = _lib().hmo_thermal_relief_f32 if dtype == np.float32 else _lib().hmo_thermal_relief_f64
    S = C.c_float if dtype == np.float32 else C.c_double
    rc = fn(int(rule), _p(z), nx, ny, _p(talus), S(sigma_inf), S(sigma_sup), int(iterations), _p(mask))
    if rc:
        raise ValueError("oracle thermal_relief rejected its arguments (status %d)" % rc)
    return z


def ref_thermal_relief(rule, z, talus=None, iterations=10, sigma_inf=0.5, sigma_sup=0.0, mask=None):
    """thermal_flatten / _inflate / _rib driven over the reference's kernel text."""
    z = _grid(z, np.float32).copy()
    ny, nx = z.shape
    talus = None if talus is None else _grid(talus, np.float32)
    mask = None if mask is None else _grid(mask, np.float32)
    rc = _ref().ref_thermal_relief(int(rule), _p(z), nx, ny, _p(talus), C.c_float(sigma_inf), C.c_float(sigma_sup),
                                   int(iterations), _p(mask))
    if rc:
        raise ValueError("ref thermal_relief rejected its arguments (status %d)" % rc)
    return z


def flow_simulation_viscous(z, water_height, depth_map, iterations, dt=0.5, dry_out_ratio=0.0, viscosity=1.0,
                            power=2.5, dtype=np.float32):
    """Oracle flow_simulation_viscous (flow_simulation.cpp:112-157); returns the water depth."""
    z = _grid(z, dtype)
    ny, nx = z.shape
    dm = _grid(depth_map, dtype)
    out = np.empty_like(z)
    fn = _lib().hmo_flow_simulation_viscous_f32 if dtype == np.float32 else _lib().hmo_flow_simulation_viscous_f64
    S = C.c_float if dtype == np.float32 else C.c_double
    rc = fn(_p(z), nx, ny, S(water_height), _p(dm), int(iterations), S(dt), S(dry_out_ratio), S(viscosity), S(power),
            _p(out))
    if rc:
        raise ValueError("oracle flow_simulation_viscous rejected its arguments (status %d)" % rc)
    return out


def ref_flow_simulation_viscous(z, water_height, depth_map, iterations, dt=0.5, dry_out_ratio=0.0, viscosity=1.0,
                                power=2.5):
    """flow_simulation.cpp:112-157 driven over the reference's shallow_viscous_flow.cl."""
    z = _grid(z, np.float32)
    ny, nx = z.shape
    dm = _grid(depth_map, np.float32)
    out = np.empty_like(z)
    rc = _ref().ref_flow_simulation_viscous(_p(z), nx, ny, C.c_float(water_height), _p(dm), int(iterations),
                                            C.c_float(dt), C.c_float(dry_out_ratio), C.c_float(viscosity),
                                            C.c_float(power), _p(out))
    if rc:
        raise ValueError("ref flow_simulation_viscous rejected its arguments (status %d)" % rc)
    return out


RIDGE, SCREE, SCHOTT, OLSEN = 0, 1, 2, 3


def thermal_sibling(rule, z, talus, iterations, zmax=None, intensity=0.2, deposition=False, mask=None,
                    dtype=np.float32):
    """Oracle ridge / scree / schott / olsen; returns (z, deposition map or None)."""
    z = _grid(z, dtype).copy()
    ny, nx = z.shape
    talus = _grid(talus, dtype)
    zmax = None if zmax is None else _grid(zmax, dtype)
    mask = None if mask is None else _grid(mask, dtype)
    depo = _out(z, deposition)
    fn = _lib().hmo_thermal_sibling_f32 if dtype == np.float32 else _lib().hmo_thermal_sibling_f64
    S = C.c_float if dtype == np.float32 else C.c_double
    rc = fn(int(rule), _p(z), nx, ny, _p(talus), _p(zmax), S(intensity), int(iterations), _p(depo), _p(mask))
    if rc:
        raise ValueError("oracle thermal_sibling rejected its arguments (status %d)" % rc)
    return z, depo


def ref_thermal_sibling(rule, z, talus, iterations, zmax=None, intensity=0.2, deposition=False, mask=None):
    """The reference's thermal_ridge / _scree / _schott / _olsen kernel text, Jacobi form."""
    z = _grid(z, np.float32).copy()
    ny, nx = z.shape
    talus = _grid(talus, np.float32)
    zmax = None if zmax is None else _grid(zmax, np.float32)
    mask = None if mask is None else _grid(mask, np.float32)
    depo = _out(z, deposition)
    rc = _ref().ref_thermal_sibling(int(rule), _p(z), nx, ny, _p(talus), _p(zmax), C.c_float(intensity),
                                    int(iterations), _p(depo), _p(mask))
    if rc:
        raise ValueError("ref thermal_sibling rejected its arguments (status %d)" % rc)
    return z, depo


def flow_simulation(z, water_height, depth_map, iterations, dt=0.5, flux_diffusion=True,
                    flux_diffusion_strength=0.01, dry_out_ratio=0.0, dtype=np.float32):
    """Oracle flow_simulation; returns the water depth."""
    z = _grid(z, dtype)
    ny, nx = z.shape
    dm = _grid(depth_map, dtype)
    out = np.empty_like(z)
    fn = _lib().hmo_flow_simulation_f32 if dtype == np.float32 else _lib().hmo_flow_simulation_f64
    S = C.c_float if dtype == np.float32 else C.c_double
    rc = fn(_p(z), nx, ny, S(water_height), _p(dm), int(iterations), S(dt), int(bool(flux_diffusion)),
            S(flux_diffusion_strength), S(dry_out_ratio), _p(out))
    if rc:
        raise ValueError("oracle flow_simulation rejected its arguments (status %d)" % rc)
    return out


def ref_flow_simulation(z, water_height, depth_map, iterations, dt=0.5, flux_diffusion=True,
                        flux_diffusion_strength=0.01, dry_out_ratio=0.0):
    """The reference's flow and water pass kernel text driven as flow_simulation."""
    z = _grid(z, np.float32)
    ny, nx = z.shape
    dm = _grid(depth_map, np.float32)
    out = np.empty_like(z)
    rc = _ref().ref_flow_simulation(_p(z), nx, ny, C.c_float(water_height), _p(dm), int(iterations),
                                    C.c_float(dt), int(bool(flux_diffusion)), C.c_float(flux_diffusion_strength),
                                    C.c_float(dry_out_ratio), _p(out))
    if rc:
        raise ValueError("ref flow_simulation rejected its arguments (status %d)" % rc)
    return out


def sample_linear_mirror(s, x, y):
    s = _grid(s, np.float32)
    ny, nx = s.shape
    return float(_lib().hmo_sample_linear_mirror_f32(_p(s), nx, ny, float(x), float(y)))


def ref_thermal(z, talus, iterations, bedrock=None, mask=None, deposition=False):
    """The reference's thermal / thermal_with_bedrock kernel text, Jacobi form."""
    z = _grid(z, np.float32).copy()
    ny, nx = z.shape
    if np.isscalar(talus):
        talus = np.full_like(z, talus)
    talus = _grid(talus, np.float32)
    bedrock = None if bedrock is None else _grid(bedrock, np.float32)
    mask = None if mask is None else _grid(mask, np.float32)
    depo = _out(z, deposition)
    rc = _ref().ref_thermal(_p(z), nx, ny, _p(talus), int(iterations), _p(bedrock), _p(depo), _p(mask))
    if rc:
        raise ValueError("ref thermal rejected its arguments (status %d)" % rc)
    return z, depo


def ref_thermal_auto_bedrock(z, talus, iterations, deposition=False):
    z = _grid(z, np.float32).copy()
    ny, nx = z.shape
    if np.isscalar(talus):
        talus = np.full_like(z, talus)
    talus = _grid(talus, np.float32)
    depo = _out(z, deposition)
    rc = _ref().ref_thermal_auto_bedrock(_p(z), nx, ny, _p(talus), int(iterations), _p(depo))
    if rc:
        raise ValueError("ref thermal_auto_bedrock rejected its arguments (status %d)" % rc)
    return z, depo


def ref_vpipes(z, params: VpipesParams, rain_map=None):
    z = _grid(z, np.float32).copy()
    ny, nx = z.shape
    rain = None if rain_map is None else _grid(rain_map, np.float32)
    outs = [np.empty_like(z) for _ in range(4)]
    rc = _ref().ref_vpipes(_p(z), nx, ny, C.byref(params), _p(rain), *[_p(o) for o in outs])
    if rc:
        raise ValueError("ref vpipes rejected its arguments (status %d)" % rc)
    return (z, *outs)


def num_threads() -> int:
    return int(_lib().hmo_num_threads())
