"""The C++ drop-in layer (include/highmap_b200/hmap_gpu.hpp): a caller
written against HighMap's hmap::gpu API, built with g++ and linked to
libhm_erosion.so, produces the oracle's results."""
import os
import subprocess

import numpy as np
import pytest

from highmap_b200.inputs import fbm
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def example(built_lib, tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("cpp") / "compat_example")
    libdir = os.path.dirname(built_lib)
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "compat_example.cpp"), "-L", libdir, "-lhm_erosion",
                    "-Wl,-rpath," + libdir, "-o", exe], check=True)
    return exe


def _run(exe, mode, z, tmp_path):
    ny, nx = z.shape
    src = tmp_path / "in.f32"
    z.tofile(src)
    prefix = str(tmp_path / "out")
    r = subprocess.run([exe, mode, str(nx), str(ny), str(src), prefix], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr

    def load(name):
        return np.fromfile(prefix + "_" + name + ".f32", dtype=np.float32).reshape(ny, nx)
    return load


def test_thermal(gpu, example, tmp_path):
    z = fbm(160, 96, seed=1)
    load = _run(example, "thermal", z, tmp_path)
    want, depo = po.thermal(z, np.full_like(z, 1 / 160), 50, bedrock=(0.3 * z).astype(np.float32),
                            deposition=True)
    assert np.array_equal(load("z"), want)
    assert np.array_equal(load("depo"), depo)


def test_config1_through_cpp(gpu, example, tmp_path):
    """The thermal benchmark configuration (256^2 fBm seed 1, talus 1/256,
    100 iterations) through hmap::gpu::thermal(Array&, float, ...)."""
    z = fbm(256, 256, seed=1)
    load = _run(example, "config1", z, tmp_path)
    want, depo = po.thermal(z, np.float32(1 / 256), 100, deposition=True)
    assert np.array_equal(load("z"), want)
    assert np.array_equal(load("depo"), depo)


def test_thermal_mask(gpu, example, tmp_path):
    z = fbm(128, 128, seed=4)
    load = _run(example, "thermal_mask", z, tmp_path)
    want, depo = po.thermal(z, np.full_like(z, 1 / 128), 50, mask=np.full_like(z, 0.25), deposition=True)
    assert np.array_equal(load("z"), want)
    assert np.array_equal(load("depo"), depo)


def test_thermal_scalar(gpu, example, tmp_path):
    z = fbm(100, 70, seed=3)
    load = _run(example, "thermal_scalar", z, tmp_path)
    want, _ = po.thermal(z, np.float32(0.1 / 100), 60)
    assert np.array_equal(load("z"), want)


def test_auto_bedrock(gpu, example, tmp_path):
    z = fbm(120, 90, seed=5)
    load = _run(example, "auto_bedrock", z, tmp_path)
    want, depo = po.thermal_auto_bedrock(z, np.full_like(z, np.float32(0.5) / np.float32(120)), 40,
                                         deposition=True)
    assert np.array_equal(load("z"), want)
    assert np.array_equal(load("depo"), depo)


def test_auto_bedrock_mask(gpu, example, tmp_path):
    z = fbm(88, 64, seed=6)
    load = _run(example, "auto_bedrock_mask", z, tmp_path)
    zf, depo = po.thermal_auto_bedrock(z, np.full_like(z, np.float32(0.5) / np.float32(88)), 40, deposition=True)
    m = np.full_like(z, 0.75)
    want = (z * (np.float32(1) - m)).astype(np.float32) + (zf * m).astype(np.float32)
    assert np.array_equal(load("z"), want)
    assert np.array_equal(load("depo"), depo)


def test_flow_simulation(gpu, example, tmp_path):
    z = fbm(90, 70, seed=8)
    load = _run(example, "flow", z, tmp_path)
    dm = (np.float32(1) - z).astype(np.float32)
    want = po.flow_simulation(z, 0.01, dm, 50, dt=0.5, flux_diffusion=True, flux_diffusion_strength=0.01,
                              dry_out_ratio=0.05)
    assert np.array_equal(load("water"), want)


@pytest.mark.parametrize("mode", ["ridge", "scree", "schott", "olsen"])
def test_sibling_stencils(gpu, example, tmp_path, mode):
    z = fbm(72, 60, seed=9)
    load = _run(example, mode, z, tmp_path)
    talus = np.full_like(z, np.float32(0.5) / np.float32(72))
    zmax = (z + np.float32(0.2)).astype(np.float32)
    mask = np.full_like(z, 0.6) if mode in ("scree", "olsen") else None
    rule = {"ridge": po.RIDGE, "scree": po.SCREE, "schott": po.SCHOTT, "olsen": po.OLSEN}[mode]
    want, depo = po.thermal_sibling(rule, z, talus, 20, zmax=zmax, intensity=0.2, deposition=mode != "olsen",
                                    mask=mask)
    assert np.array_equal(load("z"), want)
    if mode != "olsen":
        assert np.array_equal(load("depo"), depo)


def test_sediment_deposition(gpu, example, tmp_path):
    z = fbm(80, 64, seed=12)
    load = _run(example, "deposition", z, tmp_path)
    talus = np.full_like(z, np.float32(0.5) / np.float32(80))
    want, depo = po.sediment_deposition(z, talus, 0.02, 4, 8)
    assert np.array_equal(load("z"), want)
    assert np.array_equal(load("depo"), depo)


def test_sediment_layer(gpu, example, tmp_path):
    z = fbm(80, 64, seed=13)
    load = _run(example, "layer", z, tmp_path)
    tl = np.full_like(z, np.float32(0.5) / np.float32(80))
    tu = np.full_like(z, np.float32(4.0) / np.float32(80))
    want, depo = po.sediment_layer(z, tl, tu, 20, True)
    assert np.array_equal(load("z"), want)
    assert np.array_equal(load("depo"), depo)


@pytest.mark.parametrize("mode", ["flatten", "inflate", "rib"])
def test_thermal_relief(gpu, example, tmp_path, mode):
    z = fbm(72, 56, seed=14)
    load = _run(example, mode, z, tmp_path)
    talus = np.full_like(z, np.float32(0.6) / np.float32(72))
    if mode == "flatten":
        want = po.thermal_relief(po.FLATTEN, z, talus, 12, 0.5, 0.2)
    elif mode == "inflate":
        want = po.thermal_relief(po.INFLATE, z, talus, 12, mask=np.full_like(z, 0.5))
    else:
        want = po.thermal_relief(po.RIB, z, None, 6)
    assert np.array_equal(load("z"), want)


def test_flow_simulation_viscous(gpu, example, tmp_path):
    z = fbm(128, 96, seed=15)
    load = _run(example, "viscous", z, tmp_path)
    want = po.flow_simulation_viscous(z, 0.05, np.ones_like(z), 40)
    got = load("d")
    assert np.abs(got - want).max() <= 1e-3 * float(want.max())


def test_vpipes(gpu, example, tmp_path):
    z = fbm(96, 64, seed=2)
    load = _run(example, "vpipes", z, tmp_path)
    p = po.VpipesParams.make(iterations=25, flux_diffusion=0)
    wz, wd, ws, _, _ = po.vpipes(z, p)
    rng = float(z.max() - z.min())
    assert np.abs(load("z") - wz).max() <= 1e-3 * rng
    assert np.abs(load("sediment") - ws).max() <= 1e-3 * rng
    assert np.abs(load("water") - wd).max() <= 1e-3 * float(wd.max())
