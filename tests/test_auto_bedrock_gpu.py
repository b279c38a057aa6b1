"""GPU parity of thermal_auto_bedrock against the oracle, through the C-ABI.

The reference kernel (thermal.cl:102-145, driven by thermal_gpu.cpp:98-152)
keeps a bedrock grid that the GPU path folds away (a cell's bedrock after a
step equals its new value); these tests hold that folding to bit-exact
equality with the oracle, which keeps the grid as the reference does.
"""
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


def _blend(z0, z, m):
    """lerp(z0, z, mask) in fp32, one rounding per operation
    (operator.hpp:405-418 through math.cpp:183-195)."""
    one = np.float32(1)
    return (z0 * (one - m)).astype(np.float32) + (z * m).astype(np.float32)


def test_golden(gpu):
    g = dict(np.load(os.path.join(GOLDEN, "thermal_auto_bedrock.npz")))
    z = g["z"].copy()
    depo = np.empty_like(z)
    gpu.thermal_auto_bedrock(z, g["talus"], int(g["iterations"]), deposition_map=depo)
    _assert_parity(z, g["out_z"], g["z"])
    _assert_parity(depo, g["out_depo"], g["z"])


@pytest.mark.parametrize("time_block", [1, 0, 2, 3, 8])
@pytest.mark.parametrize("shape", [(256, 256), (130, 257), (9, 300), (3, 3)])
@pytest.mark.parametrize("variant", ["map", "scalar", "mask"])
def test_against_oracle(gpu, shape, variant, time_block):
    ny, nx = shape
    z0 = fbm(nx, ny, seed=4)
    talus = ((0.2 + fbm(nx, ny, seed=5)) / nx).astype(np.float32)
    iters = 29
    if variant == "scalar":
        talus_arg = np.float32(0.7 / nx)
        talus_o = np.full_like(z0, talus_arg)
    else:
        talus_arg = talus_o = talus
    want_z, want_d = po.thermal_auto_bedrock(z0, talus_o, iters, deposition=True)
    z = z0.copy()
    depo = np.empty_like(z)
    mask = None
    if variant == "mask":
        mask = fbm(nx, ny, seed=6)
        want_z = _blend(z0, want_z, mask)
    gpu.thermal_auto_bedrock(z, float(talus_arg) if variant == "scalar" else talus_arg, iters,
                             deposition_map=depo, mask=mask, time_block=time_block)
    _assert_parity(z, want_z, z0)
    _assert_parity(depo, want_d, z0)


@pytest.mark.parametrize("iters", [0, 1, 2, 9])
@pytest.mark.parametrize("time_block", [1, 4])
def test_few_iterations(gpu, iters, time_block):
    """The first step is special (its bedrock floor is -FLT_MAX) and may fall
    inside a temporally blocked launch of any depth."""
    z0 = fbm(96, 80, seed=11)
    talus = np.full_like(z0, 1.0 / 96)
    want_z, want_d = po.thermal_auto_bedrock(z0, talus, iters, deposition=True)
    z = z0.copy()
    depo = np.empty_like(z)
    gpu.thermal_auto_bedrock(z, talus, iters, deposition_map=depo, time_block=time_block)
    _assert_parity(z, want_z, z0)
    _assert_parity(depo, want_d, z0)


def test_nan_cells(gpu):
    """Cells that start NaN fail the bedrock gate and never change; their
    neighbours see a zero exchange from them."""
    z0 = fbm(64, 48, seed=12)
    z0[10, 20] = np.nan
    z0[30, 5] = np.nan
    talus = np.full_like(z0, 0.5 / 64)
    want_z, want_d = po.thermal_auto_bedrock(z0, talus, 17, deposition=True)
    z = z0.copy()
    depo = np.empty_like(z)
    gpu.thermal_auto_bedrock(z, talus, 17, deposition_map=depo)
    assert np.isnan(z[10, 20]) and np.isnan(z[30, 5])
    _assert_parity(z, want_z, z0)
    _assert_parity(depo, want_d, z0)


def test_only_deposits(gpu):
    """Interior cells never drop below their input (the reference's
    max(..., z_init)); the deposition map is therefore z - z0 inside."""
    z0 = fbm(200, 150, seed=13)
    z = z0.copy()
    depo = np.empty_like(z)
    gpu.thermal_auto_bedrock(z, 0.3 / 200, 40, deposition_map=depo)
    inner = (slice(1, -1), slice(1, -1))
    assert (z[inner] >= z0[inner]).all()
    assert np.array_equal(depo[inner], (z - z0)[inner])


def test_device_api_matches_host_api(gpu):
    import torch
    z0 = fbm(300, 200, seed=14)
    talus = ((0.5 + fbm(300, 200, seed=15)) / 300).astype(np.float32)
    mask = fbm(300, 200, seed=16)
    z_h = z0.copy()
    d_h = np.empty_like(z0)
    gpu.thermal_auto_bedrock(z_h, talus, 25, deposition_map=d_h, mask=mask)
    dev = torch.device("cuda", 0)
    z_d = torch.from_numpy(z0.copy()).to(dev)
    d_d = torch.empty_like(z_d)
    gpu.thermal_auto_bedrock_device(z_d, torch.from_numpy(talus).to(dev), 25, deposition_map=d_d,
                                    mask=torch.from_numpy(mask).to(dev))
    torch.cuda.synchronize()
    assert np.array_equal(z_d.cpu().numpy(), z_h)
    assert np.array_equal(d_d.cpu().numpy(), d_h)


def test_full_size_band(gpu):
    """4096^2, 200 iterations: a row band checked bit-exact against the
    oracle run on the band plus a halo wider than the information reach
    (one cell per step)."""
    n, iters = 4096, 200
    z0 = fbm(n, n, seed=2)
    talus = ((0.5 + fbm(n, n, seed=3)) / n).astype(np.float32)
    z = z0.copy()
    gpu.thermal_auto_bedrock(z, talus, iters)
    r0, r1 = 0, 256  # the band starts at the top border so its edge rule is the full grid's
    h = iters + 8
    want, _ = po.thermal_auto_bedrock(z0[r0:r1 + h], talus[r0:r1 + h], iters)
    # rows < r1 (with their extrapolated borders) are unaffected by the cut edge
    assert np.array_equal(z[:r1], want[:r1])
    assert (z[1:-1, 1:-1] >= z0[1:-1, 1:-1]).all()
