"""GPU parity of the snow_simulation post-filter
(HighMap/src/hydrology/snow_simulation.cpp:140-152 and its clamp_min(s, 0):
masked thermal erosion of terrain + snow, with a talus proportional to the
slope) against the oracle, through the C-ABI.  Bit-exact, with the thermal
tolerance reported on failure."""
import os

import numpy as np
import pytest

from highmap_b200.inputs import fbm
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-4  # of the height range, thermal


def _assert_parity(got, want, z0):
    fin = np.isfinite(z0)
    rng = float(z0[fin].max() - z0[fin].min()) or 1.0
    ok = np.isfinite(want)
    err = float(np.abs(got[ok].astype(np.float64) - want[ok]).max()) if ok.any() else 0.0
    assert err <= TOL * rng, "max abs err %.3g > %.3g" % (err, TOL * rng)
    assert np.array_equal(got, want, equal_nan=True), "within tolerance (%.3g) but not bit-exact" % err


def _cover(shape, seed, scale=0.08):
    ny, nx = shape
    return (scale * fbm(nx, ny, seed=seed)).astype(np.float32)


def test_golden(gpu):
    g = dict(np.load(os.path.join(GOLDEN, "snow_post_filter.npz")))
    s = g["s"].copy()
    gpu.snow_post_filter(g["z"], s, float(g["snow_depth"]), int(g["iterations"]), float(g["thermal_talus_ratio"]))
    _assert_parity(s, g["out_s"], g["z"])


@pytest.mark.parametrize("shape", [(256, 256), (130, 257), (9, 300), (3, 3), (4, 6)])
@pytest.mark.parametrize("ratio", [0.2, 1.0])
def test_against_oracle(gpu, shape, ratio):
    ny, nx = shape
    rs = np.random.RandomState(81)
    z = fbm(nx, ny, seed=81) if min(shape) > 8 else rs.rand(ny, nx).astype(np.float32)
    s0 = _cover(shape, 82) if min(shape) > 8 else (0.1 * rs.rand(ny, nx)).astype(np.float32)
    want = po.snow_post_filter(z, s0, 0.05, 27, ratio)
    s = s0.copy()
    gpu.snow_post_filter(z, s, 0.05, 27, ratio)
    _assert_parity(s, want, z)


@pytest.mark.parametrize("iters", [0, 1, 2])
def test_few_iterations(gpu, iters):
    z = fbm(96, 80, seed=83)
    s0 = _cover(z.shape, 84)
    want = po.snow_post_filter(z, s0, 0.04, iters, 0.2)
    s = s0.copy()
    gpu.snow_post_filter(z, s, 0.04, iters, 0.2)
    _assert_parity(s, want, z)


def test_deep_and_bare_cover(gpu):
    """Snow deeper than snow_depth (mask saturates through the smooth clamp)
    and bare ground (mask 0: the cell keeps z + s as it was)."""
    z = fbm(120, 90, seed=85)
    s0 = _cover(z.shape, 86, scale=0.3)
    s0[:, :40] = 0.0
    want = po.snow_post_filter(z, s0, 0.05, 19, 0.2)
    s = s0.copy()
    gpu.snow_post_filter(z, s, 0.05, 19, 0.2)
    _assert_parity(s, want, z)
    assert (s >= 0).all()


def test_device_api_matches_host_api(gpu):
    import torch
    z = fbm(300, 200, seed=87)
    s0 = _cover(z.shape, 88)
    s_h = s0.copy()
    gpu.snow_post_filter(z, s_h, 0.05, 21, 0.3)
    dev = torch.device("cuda", 0)
    s_d = torch.from_numpy(s0.copy()).to(dev)
    gpu.snow_post_filter_device(torch.from_numpy(z).to(dev), s_d, 0.05, 21, 0.3)
    torch.cuda.synchronize()
    assert np.array_equal(s_d.cpu().numpy(), s_h)


def test_rejects_bad_arguments(gpu):
    from highmap_b200 import _lib
    z = fbm(32, 32, seed=89)
    with pytest.raises(_lib.HMError):
        gpu.snow_post_filter(z, z.copy(), 0.05, -1)
    with pytest.raises(_lib.HMError):
        gpu.snow_post_filter(np.zeros((2, 2), np.float32), np.zeros((2, 2), np.float32), 0.05, 3)


def test_full_size_band(gpu):
    """2048^2, 60 iterations: a top band checked bit-exact against the
    oracle run on the band plus a halo wider than the reach of the steps."""
    n, iters = 2048, 60
    z = fbm(n, n, seed=90)
    s0 = _cover(z.shape, 91)
    s = s0.copy()
    gpu.snow_post_filter(z, s, 0.05, iters, 0.2)
    r1, h = 128, iters + 8
    want = po.snow_post_filter(z[:r1 + h], s0[:r1 + h], 0.05, iters, 0.2)
    assert np.array_equal(s[:r1], want[:r1])
    assert (s >= 0).all()
