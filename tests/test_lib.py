"""CPU tests of the C-ABI library: it builds for sm_100a, loads, exports
every function include/hm_erosion.h declares, and rejects bad arguments
before touching a device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(re.findall(r"\b(hm_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol(built_lib):
    lib = C.CDLL(built_lib)
    declared = _declared("hm_erosion.h")
    assert declared, "no declarations parsed"
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header(built_lib):
    from highmap_b200 import _lib as L
    assert _declared("hm_erosion.h") <= set(L.EXPORTED)


def test_library_is_sm100a(built_lib):
    import subprocess
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", built_lib], capture_output=True,
                         text=True).stdout
    assert "sm_100a" in out


def test_argument_checks_without_device(built_lib):
    from highmap_b200 import _lib as L
    lib = L.lib()
    z = np.zeros((4, 4), np.float32)
    # NULL context is rejected before any CUDA call
    assert lib.hm_thermal_scalar(None, C.c_void_p(z.ctypes.data), 4, 4, C.c_float(0.1), 1, None, None,
                                 None) == L.HM_ERR_INVALID_ARGUMENT
    assert lib.hm_vpipes(None, C.c_void_p(z.ctypes.data), 4, 4, None, None, None, None, None,
                         None) == L.HM_ERR_INVALID_ARGUMENT
    assert b"NULL" in lib.hm_last_error()
    assert lib.hm_status_string(L.HM_ERR_OUT_OF_MEMORY) == b"out of device memory"
    # the callers and relatives check their context first too
    zp = C.c_void_p(z.ctypes.data)
    f = C.c_float
    calls = {
        "sediment_layer": lambda: lib.hm_sediment_layer(None, zp, 4, 4, zp, zp, 1, 1, None),
        "sediment_layer_device": lambda: lib.hm_sediment_layer_device(None, zp, 4, 4, zp, zp, 1, 1, None, None),
        "snow_post_filter": lambda: lib.hm_snow_post_filter(None, zp, zp, 4, 4, f(0.1), 1, f(0.2)),
        "snow_post_filter_device": lambda: lib.hm_snow_post_filter_device(None, zp, zp, 4, 4, f(0.1), 1, f(0.2),
                                                                          None),
        "thermal_flatten": lambda: lib.hm_thermal_flatten(None, zp, 4, 4, zp, 1, f(0.5), f(0.0), None),
        "thermal_inflate": lambda: lib.hm_thermal_inflate(None, zp, 4, 4, zp, 1, None),
        "thermal_rib": lambda: lib.hm_thermal_rib(None, zp, 4, 4, 1, None),
        "thermal_relief_device": lambda: lib.hm_thermal_relief_device(None, 4, zp, 4, 4, zp, f(0.5), f(0.0), 1, None,
                                                                      None),
        "flow_simulation_viscous": lambda: lib.hm_flow_simulation_viscous(None, zp, 4, 4, f(0.01), zp, 1, f(0.5),
                                                                          f(0.0), f(1.0), f(2.5), zp),
        "flow_simulation_viscous_device": lambda: lib.hm_flow_simulation_viscous_device(
            None, zp, 4, 4, f(0.01), zp, 1, f(0.5), f(0.0), f(1.0), f(2.5), zp, None),
    }
    for name, call in calls.items():
        assert call() == L.HM_ERR_INVALID_ARGUMENT, name
        assert b"NULL" in lib.hm_last_error(), name


def test_step_kernel_selection_without_device(built_lib):
    """The vpipes step-kernel choice is process-wide host state: every
    declared algorithm, temporal blocking (two steps per launch) included,
    is accepted and anything else refused, with no device call."""
    from highmap_b200 import _lib as L
    from highmap_b200 import gpu as G
    lib = L.lib()
    try:
        for algo in (G.VPIPES_AUTO, G.VPIPES_TILED, G.VPIPES_STREAMING, G.VPIPES_TILED_CP_ASYNC,
                     G.VPIPES_TILED_TB2):
            assert lib.hm_vpipes_set_algorithm(algo) == L.HM_OK, algo
        for bad in (-2, 4, 99):
            assert lib.hm_vpipes_set_algorithm(bad) == L.HM_ERR_INVALID_ARGUMENT, bad
            assert b"unknown algorithm" in lib.hm_last_error()
    finally:
        lib.hm_vpipes_set_algorithm(G.VPIPES_AUTO)


def test_defaults_match_reference_signature(built_lib):
    """hm_vpipes_default_params carries the defaults of
    HighMap/include/highmap/erosion.hpp:1206-1223."""
    from highmap_b200 import gpu as G
    p = G.vpipes_params()
    assert p.water_height == pytest.approx(1e-2)
    assert p.maintain_water_volume == 1
    assert p.evap_rate == pytest.approx(0.1)
    assert p.iterations == 50
    assert p.dt == pytest.approx(0.5)
    assert p.k_capacity == pytest.approx(0.5)
    assert p.k_erode == pytest.approx(0.001)
    assert p.k_depose == pytest.approx(0.01)
    assert p.k_discharge_exp == 1.0
    assert p.downcutting_max_depth_ratio == 10.0
    assert p.flux_diffusion == 1
    assert p.flux_diffusion_strength == pytest.approx(0.01)
    assert (p.gravity, p.pipe_length, p.pipe_area, p.rain_per_step, p.initial_water) == (1, 1, 1, 0, -1)


def test_no_cpu_fallback_when_library_missing(monkeypatch, tmp_path):
    from highmap_b200 import _lib as L
    monkeypatch.setattr(L, "_lib", None)
    monkeypatch.setattr(L, "LIB_PATH", str(tmp_path / "missing.so"))
    with pytest.raises(RuntimeError, match="not built"):
        L.lib()


@pytest.mark.parametrize("source", ["compat_example.cpp", "overloads.cpp"])
def test_cpp_dropin_links(built_lib, tmp_path, source):
    """Callers written against HighMap's hmap::gpu API compile against
    include/highmap_b200/hmap_gpu.hpp and link to the library: the example
    program of the GPU tests, and a file that takes the address of every
    declared overload with its exact signature (so each one is defined)."""
    import subprocess
    libdir = os.path.dirname(built_lib)
    exe = str(tmp_path / source[:-4])
    r = subprocess.run(["g++", "-std=c++17", "-O0", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "cpp", source), "-L", libdir, "-lhm_erosion",
                        "-Wl,-rpath," + libdir, "-Wl,--no-undefined", "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert os.path.exists(exe)


def test_c_abi_is_plain_c(built_lib, tmp_path):
    """include/hm_erosion.h compiles as pedantic C11 without warnings, and a C
    caller (tests/c/abi_example.c) links against the library."""
    import subprocess
    libdir = os.path.dirname(built_lib)
    exe = str(tmp_path / "abi_example")
    r = subprocess.run(["gcc", "-std=c11", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I",
                        os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "c", "abi_example.c"), "-L", libdir,
                        "-lhm_erosion", "-Wl,-rpath," + libdir, "-Wl,--no-undefined", "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
