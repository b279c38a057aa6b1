"""GPU parity of sediment_layer (HighMap/src/erosion/deposition.cpp:68-113:
talus from the terrain's gradient_talus, thermal erosion with it, then an
optional laplace post-filter) against the oracle, through the C-ABI.
Bit-exact, with the thermal tolerance reported on failure."""
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


def _limits(z, seed):
    ny, nx = z.shape
    tl = ((0.5 + fbm(nx, ny, seed=seed)) / nx).astype(np.float32)
    tu = ((3.0 + 2.0 * fbm(nx, ny, seed=seed + 1)) / nx).astype(np.float32)
    return tl, tu


@pytest.mark.parametrize("case", ["sediment_layer_post", "sediment_layer_nopost"])
def test_golden(gpu, case):
    g = dict(np.load(os.path.join(GOLDEN, case + ".npz")))
    z = g["z"].copy()
    depo = np.empty_like(z)
    gpu.sediment_layer(z, g["talus_layer"], g["talus_upper_limit"], int(g["iterations"]),
                       bool(g["apply_post_filter"]), deposition_map=depo)
    _assert_parity(z, g["out_z"], g["z"])
    _assert_parity(depo, g["out_depo"], g["z"])


@pytest.mark.parametrize("shape", [(256, 256), (130, 257), (41, 53), (40, 52), (9, 300), (3, 3), (4, 6), (7, 5)])
@pytest.mark.parametrize("post", [True, False])
def test_against_oracle(gpu, shape, post):
    """Odd and even sizes in both directions: gradient_talus pairs columns
    and rows from index 1, so the last column / row is handled differently
    for each parity."""
    ny, nx = shape
    z0 = fbm(nx, ny, seed=61) if min(shape) > 8 else np.random.RandomState(61).rand(ny, nx).astype(np.float32)
    tl, tu = _limits(z0, 62)
    want, want_d = po.sediment_layer(z0, tl, tu, 23, post)
    z = z0.copy()
    depo = np.empty_like(z)
    gpu.sediment_layer(z, tl, tu, 23, post, deposition_map=depo)
    _assert_parity(z, want, z0)
    _assert_parity(depo, want_d, z0)


@pytest.mark.parametrize("iters", [0, 1, 2])
def test_few_iterations(gpu, iters):
    z0 = fbm(96, 80, seed=63)
    tl, tu = _limits(z0, 64)
    for post in (True, False):
        want, want_d = po.sediment_layer(z0, tl, tu, iters, post)
        z = z0.copy()
        gpu.sediment_layer(z, tl, tu, iters, post)
        _assert_parity(z, want, z0)
        depo = np.empty_like(z)
        z = z0.copy()
        gpu.sediment_layer(z, tl, tu, iters, post, deposition_map=depo)
        _assert_parity(depo, want_d, z0)


def test_all_or_no_cells_steep(gpu):
    """Upper limits below and above every slope: every cell takes the
    steepened talus and a zero filter mask, or none does."""
    z0 = fbm(120, 90, seed=65)
    tl = np.full_like(z0, 0.5 / 120)
    for tu in (np.zeros_like(z0), np.full_like(z0, 10.0)):
        want, want_d = po.sediment_layer(z0, tl, tu, 17, True)
        z = z0.copy()
        depo = np.empty_like(z)
        gpu.sediment_layer(z, tl, tu, 17, True, deposition_map=depo)
        _assert_parity(z, want, z0)
        _assert_parity(depo, want_d, z0)


def test_nan_cells(gpu):
    z0 = fbm(64, 48, seed=66)
    z0[10, 21] = np.nan
    z0[31, 6] = np.nan
    tl, tu = _limits(z0, 67)
    for post in (True, False):
        want, want_d = po.sediment_layer(z0, tl, tu, 11, post)
        z = z0.copy()
        depo = np.empty_like(z)
        gpu.sediment_layer(z, tl, tu, 11, post, deposition_map=depo)
        _assert_parity(z, want, z0)
        _assert_parity(depo, want_d, z0)


def test_device_api_matches_host_api(gpu):
    import torch
    z0 = fbm(300, 200, seed=68)
    tl, tu = _limits(z0, 69)
    z_h = z0.copy()
    d_h = np.empty_like(z0)
    gpu.sediment_layer(z_h, tl, tu, 21, True, deposition_map=d_h)
    dev = torch.device("cuda", 0)
    z_d = torch.from_numpy(z0.copy()).to(dev)
    d_d = torch.empty_like(z_d)
    gpu.sediment_layer_device(z_d, torch.from_numpy(tl).to(dev), torch.from_numpy(tu).to(dev), 21, True,
                              deposition_map=d_d)
    torch.cuda.synchronize()
    assert np.array_equal(z_d.cpu().numpy(), z_h)
    assert np.array_equal(d_d.cpu().numpy(), d_h)


def test_rejects_bad_arguments(gpu):
    from highmap_b200 import _lib
    z = fbm(32, 32, seed=70)
    with pytest.raises(_lib.HMError):
        gpu.sediment_layer(z, z, z, -1)
    with pytest.raises(_lib.HMError):
        gpu.sediment_layer(np.zeros((2, 2), np.float32), np.zeros((2, 2), np.float32),
                           np.zeros((2, 2), np.float32), 3)


def test_full_size_band(gpu):
    """2048^2, 60 iterations with the post-filter: a top band checked
    bit-exact against the oracle run on the band plus a halo wider than the
    reach of the slope, the thermal steps (one cell each) and the filter."""
    n, iters = 2048, 60
    z0 = fbm(n, n, seed=71)
    tl, tu = _limits(z0, 72)
    z = z0.copy()
    depo = np.empty_like(z)
    gpu.sediment_layer(z, tl, tu, iters, True, deposition_map=depo)
    r1, h = 128, iters + 16
    want, want_d = po.sediment_layer(z0[:r1 + h], tl[:r1 + h], tu[:r1 + h], iters, True)
    assert np.array_equal(z[:r1], want[:r1])
    assert np.array_equal(depo[:r1], want_d[:r1])
    assert (depo >= 0).all()
