"""CPU tests of the oracle: pinned to the reference's kernel text.

1. Against the golden fixtures (tests/golden/, made from the reference's
   own OpenCL kernels compiled for the CPU): bit-exact wherever the oracle
   and the reference evaluate the same fp32 operations; within a tight
   tolerance where they differ by construction (the reference sums the
   water volume serially in float, the oracle in fp64).
2. Against the reference checker on fresh seeded inputs, when it is built.
3. Property tests in the style of the reference's unit tests
   (tests/src/test_smooth_cpulse.cpp and friends): flat field unchanged,
   slopes under talus unchanged, a spike relaxes symmetrically, interior
   mass conservation, no water means no erosion.
"""
import glob
import json
import os

import numpy as np
import pytest

from highmap_b200.inputs import fbm
from oracle import pyoracle as po

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def _params(g):
    return po.VpipesParams.make(**json.loads(str(g["params"])))


def test_config1_golden_digests():
    """The thermal benchmark configuration (256^2 fBm seed 1, talus 1/256,
    100 iterations): the generated input and the oracle's heights and
    deposition map have the digests of the reference text's outputs."""
    import hashlib

    def digest(a):
        return np.frombuffer(hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest(), dtype=np.uint8)
    g = _load("config1_thermal_256")
    z0 = fbm(256, 256, seed=1)
    assert np.array_equal(digest(z0), g["z_sha256"])
    z, depo = po.thermal(z0, np.float32(g["talus"]), int(g["iterations"]), deposition=True)
    assert np.array_equal(digest(z), g["out_z_sha256"])
    assert np.array_equal(digest(depo), g["out_depo_sha256"])


@pytest.mark.parametrize("name", ["thermal_uniform", "thermal_talus_map", "thermal_masked", "thermal_small_3x3",
                                  "thermal_small_5x17", "thermal_small_33x7"])
def test_thermal_golden_bit_exact(name):
    g = _load(name)
    z, depo = po.thermal(g["z"], g["talus"], int(g["iterations"]), mask=g.get("mask"), deposition=True)
    assert np.array_equal(z, g["out_z"])
    assert np.array_equal(depo, g["out_depo"])


def test_thermal_bedrock_literal_golden():
    g = _load("thermal_bedrock_literal")
    z, depo = po.thermal(g["z"], g["talus"], int(g["iterations"]), bedrock=g["bedrock"], deposition=True,
                         bedrock_mode=po.BEDROCK_LITERAL)
    assert np.array_equal(z, g["out_z"])
    assert np.array_equal(depo, g["out_depo"])


def test_thermal_auto_bedrock_golden():
    g = _load("thermal_auto_bedrock")
    z, depo = po.thermal_auto_bedrock(g["z"], g["talus"], int(g["iterations"]), deposition=True)
    assert np.array_equal(z, g["out_z"])
    assert np.array_equal(depo, g["out_depo"])


@pytest.mark.parametrize("name", ["vpipes_no_maintain", "vpipes_rain_per_step", "vpipes_exp_half"])
def test_vpipes_golden_bit_exact(name):
    g = _load(name)
    out = po.vpipes(g["z"], _params(g), rain_map=g.get("rain_map"))
    for got, key in zip(out, ("out_z", "out_water", "out_sediment", "out_u", "out_v")):
        assert np.array_equal(got, g[key]), key


@pytest.mark.parametrize("name", ["vpipes_defaults", "vpipes_rain_map"])
def test_vpipes_golden_volume_sum(name):
    """maintain_water_volume: the reference sums the depth serially in
    float (Array::sum); the oracle sums in fp64.  The outputs agree to well
    inside the 1e-3 height-range tolerance."""
    g = _load(name)
    out = po.vpipes(g["z"], _params(g), rain_map=g.get("rain_map"))
    rng = float(g["z"].max() - g["z"].min())
    assert np.abs(out[0] - g["out_z"]).max() <= 1e-4 * rng
    assert np.abs(out[1] - g["out_water"]).max() <= 1e-4 * float(g["out_water"].max())
    assert np.abs(out[2] - g["out_sediment"]).max() <= 1e-4 * rng


@pytest.mark.parametrize("name", ["flow_simulation_defaults", "flow_simulation_dry_out"])
def test_flow_simulation_golden_bit_exact(name):
    g = _load(name)
    kw = json.loads(str(g["params"]))
    out = po.flow_simulation(g["z"], depth_map=g["depth_map"], **kw)
    assert np.array_equal(out, g["out_water"])


@pytest.mark.parametrize("name,rule", [("thermal_ridge", po.RIDGE), ("thermal_scree", po.SCREE),
                                       ("thermal_schott", po.SCHOTT), ("thermal_olsen", po.OLSEN)])
def test_sibling_golden_bit_exact(name, rule):
    g = _load(name)
    kw = {}
    if "zmax" in g:
        kw["zmax"] = g["zmax"]
    if "intensity" in g:
        kw["intensity"] = float(g["intensity"])
    z, depo = po.thermal_sibling(rule, g["z"], g["talus"], int(g["iterations"]), deposition="out_depo" in g, **kw)
    assert np.array_equal(z, g["out_z"])
    if "out_depo" in g:
        assert np.array_equal(depo, g["out_depo"])


def test_sediment_deposition_golden_bit_exact():
    g = _load("sediment_deposition")
    kw = json.loads(str(g["params"]))
    z, depo = po.sediment_deposition(g["z"], g["talus"], **kw)
    assert np.array_equal(z, g["out_z"]) and np.array_equal(depo, g["out_depo"])


@pytest.mark.parametrize("case", ["sediment_layer_post", "sediment_layer_nopost"])
def test_sediment_layer_golden_bit_exact(case):
    g = _load(case)
    z, depo = po.sediment_layer(g["z"], g["talus_layer"], g["talus_upper_limit"], int(g["iterations"]),
                                bool(g["apply_post_filter"]))
    assert np.array_equal(z, g["out_z"]) and np.array_equal(depo, g["out_depo"])
    # the solve moved material in a good share of the cells
    assert 0.1 < float((depo != 0).mean()) <= 1.0


def test_snow_post_filter_golden_bit_exact():
    g = _load("snow_post_filter")
    out = po.snow_post_filter(g["z"], g["s"], float(g["snow_depth"]), int(g["iterations"]),
                              float(g["thermal_talus_ratio"]))
    assert np.array_equal(out, g["out_s"])
    assert (out >= 0).all() and not np.array_equal(out, g["s"])


@pytest.mark.parametrize("case", ["thermal_flatten", "thermal_flatten_masked", "thermal_inflate", "thermal_rib",
                                  "thermal_rib_masked"])
def test_thermal_relief_golden_bit_exact(case):
    g = _load(case)
    z = po.thermal_relief(int(g["rule"]), g["z"], g["talus"], int(g["iterations"]), float(g["sigma_inf"]),
                          float(g["sigma_sup"]), mask=g.get("mask"))
    assert np.array_equal(z, g["out_z"])


@pytest.mark.parametrize("case", ["flow_simulation_viscous", "flow_simulation_viscous_dry"])
def test_flow_simulation_viscous_golden_bit_exact(case):
    g = _load(case)
    out = po.flow_simulation_viscous(g["z"], float(g["water_height"]), g["depth_map"], int(g["iterations"]), 0.5,
                                     float(g["dry_out_ratio"]), float(g["viscosity"]), float(g["power"]))
    assert np.array_equal(out, g["out_d"])


def test_golden_files_present():
    names = {os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))}
    assert {"thermal_uniform", "vpipes_defaults", "vpipes_rain_per_step"} <= names


ref_only = pytest.mark.skipif(not po.ref_available(), reason="reference checker not built here")


@ref_only
@pytest.mark.parametrize("seed", [11, 12])
def test_thermal_matches_reference_text(seed):
    z = fbm(71, 53, seed=seed)
    talus = (0.5 + fbm(71, 53, seed=seed + 100)) / 71
    bed = (0.5 * z).astype(np.float32)
    for kw in (dict(), dict(bedrock=bed)):
        a, da = po.thermal(z, talus, 30, deposition=True, bedrock_mode=po.BEDROCK_LITERAL, **kw)
        b, db = po.ref_thermal(z, talus, 30, deposition=True, **kw)
        assert np.array_equal(a, b) and np.array_equal(da, db)


@ref_only
def test_vpipes_matches_reference_text():
    z = fbm(40, 56, seed=21)
    p = po.VpipesParams.make(iterations=15, maintain_water_volume=0, flux_diffusion=1, dt=0.3)
    a = po.vpipes(z, p)
    b = po.ref_vpipes(z, p)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


@ref_only
def test_flow_simulation_matches_reference_text():
    z = fbm(61, 47, seed=22)
    dm = fbm(61, 47, seed=23)
    for kw in (dict(flux_diffusion=True, dry_out_ratio=0.0), dict(flux_diffusion=False, dry_out_ratio=0.2)):
        a = po.flow_simulation(z, 0.015, dm, 35, dt=0.4, **kw)
        b = po.ref_flow_simulation(z, 0.015, dm, 35, dt=0.4, **kw)
        assert np.array_equal(a, b)


@ref_only
@pytest.mark.parametrize("rule", [0, 1, 2, 3])
def test_siblings_match_reference_text(rule):
    z = fbm(59, 41, seed=24)
    talus = ((0.3 + fbm(59, 41, seed=25)) / 59).astype(np.float32)
    zmax = (z + 0.25).astype(np.float32)
    mask = fbm(59, 41, seed=26)
    for m in (None, mask):
        a, da = po.thermal_sibling(rule, z, talus, 20, zmax=zmax, intensity=0.15, deposition=True, mask=m)
        b, db = po.ref_thermal_sibling(rule, z, talus, 20, zmax=zmax, intensity=0.15, deposition=True, mask=m)
        assert np.array_equal(a, b)
        if rule != po.OLSEN:
            assert np.array_equal(da, db)


@ref_only
def test_sediment_deposition_matches_reference_text():
    z = fbm(47, 39, seed=27)
    talus = ((0.3 + fbm(47, 39, seed=28)) / 47).astype(np.float32)
    mask = fbm(47, 39, seed=29)
    for m in (None, mask):
        a, da = po.sediment_deposition(z, talus, 0.03, 3, 6, mask=m)
        b, db = po.ref_sediment_deposition(z, talus, 0.03, 3, 6, mask=m)
        assert np.array_equal(a, b) and np.array_equal(da, db)


def test_flat_field_unchanged():
    z = np.full((20, 24), 0.5, np.float32)
    out, depo = po.thermal(z, 0.01, 50, deposition=True)
    assert np.array_equal(out, z)
    assert not depo.any()


def test_slope_below_talus_unchanged():
    ny, nx = 30, 40
    z = (np.arange(nx, dtype=np.float32)[None, :] * 0.001 + np.zeros((ny, 1), np.float32)).astype(np.float32)
    out, _ = po.thermal(z, 0.0011, 20)
    # interior unchanged; the border is extrapolated linearly, which keeps a plane
    np.testing.assert_allclose(out, z, atol=1e-6)


def test_spike_relaxes_symmetrically():
    n = 33
    z = np.zeros((n, n), np.float32)
    z[n // 2, n // 2] = 1.0
    out, _ = po.thermal(z, 0.0, 8)
    inner = out[2:-2, 2:-2]
    assert np.allclose(inner, inner.T, atol=1e-7)
    assert np.allclose(inner, inner[::-1, :], atol=1e-7)
    assert out[n // 2, n // 2] < 1.0


def test_interior_mass_conserved_uniform_talus():
    """With a uniform talus every exchange is antisymmetric between the two
    cells, so the sum over cells far from the border (where the border
    copy rule cannot reach in a few steps) changes only by rounding."""
    n = 64
    z = np.zeros((n, n), np.float32)
    z[24:40, 24:40] = fbm(16, 16, seed=4)
    out, _ = po.thermal(z, 0.001, 6, dtype=np.float64)
    assert abs(out.sum() - z.astype(np.float64).sum()) < 1e-9


def test_vpipes_dry_leaves_terrain():
    z = fbm(32, 24, seed=5)
    p = po.VpipesParams.make(iterations=10, water_height=1e-2, initial_water=0.0, maintain_water_volume=0)
    zo, d, s, u, v = po.vpipes(z, p)
    assert np.array_equal(zo, z)
    assert not s.any() and not d.any() and not u.any() and not v.any()


def test_sampler_half_texel_shift():
    """At zero velocity the linear sampler blends (i-1, i) with weights 1/2:
    texel centres are at k + 0.5 (hydraulic_vpipes.cl:207-208)."""
    s = np.arange(12, dtype=np.float32).reshape(3, 4)
    assert po.sample_linear_mirror(s, 2.0, 1.5) == pytest.approx(0.5 * (s[1, 1] + s[1, 2]))
    # mirrored repeat at the left edge: texel -1 reads texel 0
    assert po.sample_linear_mirror(s, 0.0, 1.5) == pytest.approx(s[1, 0])
    # far outside: mirror with period 2 * width
    assert po.sample_linear_mirror(s, 8.5 + 0.0, 1.5) == pytest.approx(po.sample_linear_mirror(s, 0.5, 1.5))


def test_float_vs_double_thermal_error_small():
    z = fbm(64, 64, seed=1)
    a, _ = po.thermal(z, 1 / 64, 100)
    b, _ = po.thermal(z.astype(np.float64), 1 / 64, 100, dtype=np.float64)
    assert np.abs(a - b).max() <= 1e-4 * float(z.max() - z.min())


def test_float_vs_double_vpipes_error_small():
    z = fbm(48, 48, seed=2)
    p = po.VpipesParams.make(iterations=30)
    a = po.vpipes(z, p)
    b = po.vpipes(z.astype(np.float64), p, dtype=np.float64)
    assert np.abs(a[0] - b[0]).max() <= 1e-3 * float(z.max() - z.min())


def test_fast_water_case_exceeds_staged_radius():
    """The fast-water case of the GPU launch-shape tests moves sediment
    further than the largest staged advection radius (3 cells), so those
    tests exercise the kernel's exact slow path."""
    fast = dict(maintain_water_volume=0, flux_diffusion=1, dt=0.5, gravity=40.0, initial_water=0.05, iterations=12)
    z0 = fbm(333, 300, seed=5)
    out = po.vpipes(z0, po.VpipesParams.make(**fast))
    reach = fast["dt"] * np.maximum(np.abs(out[3]), np.abs(out[4]))
    assert float(reach.max()) > 3.5


@ref_only
@pytest.mark.parametrize("shape", [(41, 53), (40, 52), (3, 3), (4, 6), (7, 5)])
def test_sediment_layer_matches_reference_text(shape):
    ny, nx = shape
    z = fbm(nx, ny, seed=31) if min(shape) > 8 else np.random.RandomState(31).rand(ny, nx).astype(np.float32)
    tl = np.full_like(z, 0.5 / nx)
    tu = ((3.0 + 2.0 * fbm(nx, ny, seed=32)) / nx).astype(np.float32)
    for post in (True, False):
        a, da = po.sediment_layer(z, tl, tu, 12, post)
        b, db = po.ref_sediment_layer(z, tl, tu, 12, post)
        assert np.array_equal(a, b) and np.array_equal(da, db)


@ref_only
@pytest.mark.parametrize("shape", [(41, 53), (3, 3), (4, 6)])
def test_snow_post_filter_matches_reference_text(shape):
    ny, nx = shape
    rs = np.random.RandomState(35)
    z = fbm(nx, ny, seed=35) if min(shape) > 8 else rs.rand(ny, nx).astype(np.float32)
    s = (0.1 * rs.rand(ny, nx)).astype(np.float32)
    for ratio in (0.2, 1.0):
        a = po.snow_post_filter(z, s, 0.05, 15, ratio)
        b = po.ref_snow_post_filter(z, s, 0.05, 15, ratio)
        assert np.array_equal(a, b)


@ref_only
@pytest.mark.parametrize("rule", [4, 5, 6])
@pytest.mark.parametrize("shape", [(41, 53), (5, 5), (6, 9)])
def test_thermal_relief_matches_reference_text(rule, shape):
    ny, nx = shape
    rs = np.random.RandomState(40 + rule)
    z = fbm(nx, ny, seed=41) if min(shape) > 8 else rs.rand(ny, nx).astype(np.float32)
    talus = np.full_like(z, 0.6 / nx)
    mask = rs.rand(ny, nx).astype(np.float32)
    for m in (None, mask):
        a = po.thermal_relief(rule, z, talus, 9, 0.5, 0.3, mask=m)
        b = po.ref_thermal_relief(rule, z, talus, 9, 0.5, 0.3, mask=m)
        assert np.array_equal(a, b, equal_nan=True)


@ref_only
@pytest.mark.parametrize("shape", [(41, 53), (1, 7), (6, 1), (64, 96)])
def test_flow_simulation_viscous_matches_reference_text(shape):
    ny, nx = shape
    rs = np.random.RandomState(61)
    z = fbm(nx, ny, seed=61) if min(shape) > 8 else rs.rand(ny, nx).astype(np.float32)
    dm = fbm(nx, ny, seed=62) if min(shape) > 8 else rs.rand(ny, nx).astype(np.float32)
    for dry, power in ((0.0, 2.5), (0.2, 1.5)):
        a = po.flow_simulation_viscous(z, 0.04, dm, 25, 0.5, dry, 1.3, power)
        b = po.ref_flow_simulation_viscous(z, 0.04, dm, 25, 0.5, dry, 1.3, power)
        assert np.array_equal(a, b, equal_nan=True)


@ref_only
def test_golden_fixtures_regenerate_bit_exact(tmp_path):
    """Every committed fixture is exactly what tests/golden/make_golden.py
    makes from the reference's kernel text: regenerate all groups into a
    temporary directory and compare array by array."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    mg.OUT_DIR = str(tmp_path)
    for group in mg.GROUPS.values():
        group()
    made = sorted(os.path.basename(p) for p in glob.glob(os.path.join(str(tmp_path), "*.npz")))
    committed = sorted(os.path.basename(p) for p in glob.glob(os.path.join(GOLDEN, "*.npz")))
    assert made == committed
    for name in made:
        a = np.load(os.path.join(str(tmp_path), name))
        b = np.load(os.path.join(GOLDEN, name))
        assert sorted(a.files) == sorted(b.files), name
        for k in a.files:
            assert a[k].dtype == b[k].dtype, (name, k)
            floating = np.issubdtype(a[k].dtype, np.floating)
            assert np.array_equal(a[k], b[k], equal_nan=floating), (name, k)
